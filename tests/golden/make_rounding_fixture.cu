// Generates tests/golden/rounding_sr.bin: outputs of the B200's stochastic-
// rounding conversions cvt.rs.f16x2.f32 and cvt.rs.bf16x2.f32 (the 16-bit
// field storages' rounding), against which the oracle's restatement is
// checked on the CPU (tests/test_oracle_round16.py).
//   nvcc -gencode arch=compute_100a,code=sm_100a -O2 -o mk make_rounding_fixture.cu && ./mk rounding_sr.bin
// Cases: every single-bit random word against fractions j/16 of the FP16 unit
// at [1, 2); 16384 uniform random values in [0, 2) with random words; and
// every random case (of 2^20) with an input below FP16's normal range.
// File: int32 n, then n floats a, n floats b, n u32 rbits, n u32 f16x2, n u32 bf16x2
// (a is converted into the high half, b into the low half).
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>
#include <cuda_runtime.h>

__global__ void k_rs(const float* a, const float* b, const unsigned* rb, unsigned* o16, unsigned* obf, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned d, e;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a[i]), "f"(b[i]), "r"(rb[i]));
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(e) : "f"(a[i]), "f"(b[i]), "r"(rb[i]));
    o16[i] = d;
    obf[i] = e;
}

int main(int argc, char** argv) {
    std::vector<float> a, b;
    std::vector<unsigned> r;
    for (int bit = -1; bit < 32; ++bit)
        for (int j = 0; j < 16; ++j) {
            const uint32_t ua = 0x3f800000u + (uint32_t)(j << 9), ub = 0x3f800000u + (uint32_t)((15 - j) << 9);
            float fa, fb;
            memcpy(&fa, &ua, 4);
            memcpy(&fb, &ub, 4);
            a.push_back(fa);
            b.push_back(fb);
            r.push_back(bit < 0 ? 0u : (1u << bit));
        }
    std::mt19937 g(7);
    std::uniform_real_distribution<float> u(0.0f, 2.0f);
    for (int i = 0; i < (1 << 20); ++i) {
        const float fa = u(g), fb = u(g);
        const unsigned rv = g();
        if (i < 16384 || fa < 6.103515625e-05f || fb < 6.103515625e-05f) {
            a.push_back(fa);
            b.push_back(fb);
            r.push_back(rv);
        }
    }
    const int n = (int)a.size();
    float *da, *db;
    unsigned *dr, *o1, *o2;
    cudaMalloc(&da, n * 4);
    cudaMalloc(&db, n * 4);
    cudaMalloc(&dr, n * 4);
    cudaMalloc(&o1, n * 4);
    cudaMalloc(&o2, n * 4);
    cudaMemcpy(da, a.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(db, b.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dr, r.data(), n * 4, cudaMemcpyHostToDevice);
    k_rs<<<(n + 255) / 256, 256>>>(da, db, dr, o1, o2, n);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        printf("cuda error %s\n", cudaGetErrorString(e));
        return 1;
    }
    std::vector<unsigned> h1(n), h2(n);
    cudaMemcpy(h1.data(), o1, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(h2.data(), o2, n * 4, cudaMemcpyDeviceToHost);
    FILE* f = fopen(argc > 1 ? argv[1] : "rounding_sr.bin", "wb");
    fwrite(&n, 4, 1, f);
    fwrite(a.data(), 4, n, f);
    fwrite(b.data(), 4, n, f);
    fwrite(r.data(), 4, n, f);
    fwrite(h1.data(), 4, n, f);
    fwrite(h2.data(), 4, n, f);
    fclose(f);
    printf("%d cases\n", n);
    return 0;
}
