// Drop-in for kunpBFV's include/Utils.cuh: the compat classes plus the two
// printing helpers the reference's drivers call (bfv_demo.cu), written here
// for this header: print_host__array prints the first 11 values of two host
// arrays, print_device_array_max copies up to max_size values of a device array
// to the host and prints them (include/Utils.cuh:350-362, 434-448 define the
// originals).
#pragma once
#include <cstdio>
#include <vector>

#include "../../kbfv_compat_global.hpp"

inline void print_host__array(uint64_tt* data, uint64_tt* data2, int slots) {
    const int n = slots < 11 ? slots : 11;
    std::printf("mes1 = [ ");
    for (int i = 0; i < n; ++i) std::printf("%llu ", data[i]);
    std::printf(" ]\nmes2 = [ ");
    for (int i = 0; i < n; ++i) std::printf("%llu ", data2[i]);
    std::printf(" ]\n");
}

inline void print_device_array_max(uint64_tt* data, int slots, const char* vname, int max_size) {
    const int n = slots < max_size ? slots : max_size;
    std::vector<uint64_tt> h(n > 0 ? n : 0);
    cudaDeviceSynchronize();
    if (n > 0) cudaMemcpy(h.data(), data, sizeof(uint64_tt) * n, cudaMemcpyDeviceToHost);
    std::printf("%s = [", vname);
    for (int i = 0; i < n; ++i) std::printf("%05llu, ", h[i]);
    std::printf("]\n");
}
