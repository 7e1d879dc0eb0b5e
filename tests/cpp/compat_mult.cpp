// A kunpBFV-style driver (the flow of the reference's correct_mult.cu) written
// against include/kbfv_compat.hpp: encode, encrypt, multiply + relinearise,
// multiply by a plaintext, decrypt, decode; exits non-zero on any wrong slot.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "kbfv_compat.hpp"

using namespace kbfv_compat;

int main(int argc, char** argv) {
    size_t poly_modulus_degree = argc > 1 ? (size_t)atol(argv[1]) : 16384;
    BFVContext context(poly_modulus_degree);
    BFVScheme scheme(context);
    SecretKey sk(context);
    scheme.mallocMemory();
    scheme.addEncKey(sk);
    scheme.addMultKey_23(sk);
    scheme.addLeftRotKey_23(sk, 1);
    scheme.addLeftRotKey_23(sk, 2);

    const int N = (int)context.N, L = context.L, slots = context.slots;
    const uint64_tt t = context.plain_modulus;
    std::vector<uint64_tt> mes1(slots), mes2(slots);
    srand(7);
    for (int i = 0; i < slots; ++i) {
        mes1[i] = (uint64_tt)rand() % t;
        mes2[i] = (uint64_tt)rand() % t;
    }
    uint64_tt *d_msg1, *d_msg2, *d_dec;
    check_cuda(cudaMalloc(&d_msg1, sizeof(uint64_tt) * slots));
    check_cuda(cudaMalloc(&d_msg2, sizeof(uint64_tt) * slots));
    check_cuda(cudaMalloc(&d_dec, sizeof(uint64_tt) * slots));
    check_cuda(cudaMemcpy(d_msg1, mes1.data(), sizeof(uint64_tt) * slots, cudaMemcpyHostToDevice));
    check_cuda(cudaMemcpy(d_msg2, mes2.data(), sizeof(uint64_tt) * slots, cudaMemcpyHostToDevice));

    Plaintext plain1(N, L, L, slots), plain2(N, L, L, slots), plain1_ntt(N, L, L, slots);
    Ciphertext c1(N, L, L, slots), c2(N, L, L, slots);
    context.encode(d_msg1, plain1);
    context.encode(d_msg2, plain2);
    context.encode_ntt(d_msg1, plain1_ntt);  // d_msg1 now holds plain1's coefficients
    scheme.encryptMsg(c1, plain1);
    scheme.encryptMsg(c2, plain2);
    scheme.multAndEqual_23(c1, c2);
    scheme.multConstAndEqual(c1, plain1_ntt);

    Plaintext plain_dec(N, L, L, slots);
    scheme.decryptMsg(plain_dec, sk, c1);
    context.decode(plain_dec, d_dec);
    std::vector<uint64_tt> dec(slots);
    check_cuda(cudaMemcpy(dec.data(), d_dec, sizeof(uint64_tt) * slots, cudaMemcpyDeviceToHost));

    int bad = 0;
    for (int i = 0; i < slots; ++i) {
        const uint64_tt want = (uint64_tt)((unsigned __int128)mes1[i] * mes2[i] % t * mes1[i] % t);
        if (dec[i] != want) bad++;
    }
    // rotations: left by 1 twice equals left by 2; plaintext and constant additions
    Ciphertext c3(N, L, L, slots), c4(N, L, L, slots);
    scheme.encryptMsg(c3, plain2);
    scheme.encryptMsg(c4, plain2);
    scheme.leftRotateAndEqual_23(c3, 1);
    scheme.leftRotateAndEqual_23(c3, 1);
    scheme.leftRotateAndEqual_23(c4, 2);
    std::vector<uint64_tt> r3(slots), r4(slots), r5(slots);
    scheme.decryptMsg(plain_dec, sk, c3);
    context.decode(plain_dec, d_dec);
    check_cuda(cudaMemcpy(r3.data(), d_dec, sizeof(uint64_tt) * slots, cudaMemcpyDeviceToHost));
    scheme.decryptMsg(plain_dec, sk, c4);
    context.decode(plain_dec, d_dec);
    check_cuda(cudaMemcpy(r4.data(), d_dec, sizeof(uint64_tt) * slots, cudaMemcpyDeviceToHost));
    int moved = 0;
    for (int i = 0; i < slots; ++i) {
        if (r3[i] != r4[i]) bad++;
        if (r3[i] != mes2[i]) moved++;
    }
    if (moved == 0) bad++;  // a rotation that changed nothing
    Ciphertext c5(N, L, L, slots);
    scheme.encryptMsg(c5, plain2);
    scheme.addConstAndEqual(c5, plain1);  // plain1 holds mes1's coefficients
    scheme.addConstAndEqual(c5, (uint64_tt)5);
    scheme.decryptMsg(plain_dec, sk, c5);
    context.decode(plain_dec, d_dec);
    check_cuda(cudaMemcpy(r5.data(), d_dec, sizeof(uint64_tt) * slots, cudaMemcpyDeviceToHost));
    for (int i = 0; i < slots; ++i)
        if (r5[i] != (mes1[i] + mes2[i] + 5) % t) bad++;

    printf("N=%d slots=%d wrong=%d first: ", N, slots, bad);
    for (int i = 0; i < 4; ++i) printf("%llu ", dec[i]);
    printf("\n");
    return bad == 0 ? 0 : 1;
}
