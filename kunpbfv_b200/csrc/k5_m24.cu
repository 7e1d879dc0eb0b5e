// K5 kernels for contexts of at most 23 ciphertext primes (the MAXQ = 24 bucket)
#include "k5_kernels.cuh"

template void q2r_ntt_launch_m<24>(const DevConsts&, const uint64_t*, uint64_t*, int, cudaStream_t);
template void k5_launch_m<24>(const DevConsts&, int, const MulScratch&, uint64_t*, int, cudaStream_t);
template void bconv_mixed_launch_m<24>(const Groups&, const LaunchShape&, int, const MulScratch&, cudaStream_t);
template void k5_mixed_launch_m<24>(const Groups&, const LaunchShape&, int, const MulScratch&, cudaStream_t);
