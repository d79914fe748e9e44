// Known-answer generator for the packed stochastic-rounding conversions
// cvt.rs.f16x2.f32 and cvt.rs.bf16x2.f32 of sm_100a (with and without
// .satfinite): converts seeded (a, b, rbits) triples on the GPU.  Used by
// tests/golden/make_cvt_rs_golden.py and tests/test_gpu_storage16.py to pin
// the oracle's restatement of the rounding rule.
//
// Output file: int32 n, then a[n], b[n] (f32), rbits[n], and the four result
// arrays (f16x2, f16x2 satfinite, bf16x2, bf16x2 satfinite), uint32 each.
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>

__global__ void k(const float* a, const float* b, const uint32_t* r, uint32_t* o16, uint32_t* o16s,
                  uint32_t* ob16, uint32_t* ob16s, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t d0, d1, d2, d3;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d0) : "f"(a[i]), "f"(b[i]), "r"(r[i]));
    asm("cvt.rs.satfinite.f16x2.f32 %0, %1, %2, %3;" : "=r"(d1) : "f"(a[i]), "f"(b[i]), "r"(r[i]));
    asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d2) : "f"(a[i]), "f"(b[i]), "r"(r[i]));
    asm("cvt.rs.satfinite.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d3) : "f"(a[i]), "f"(b[i]), "r"(r[i]));
    o16[i] = d0; o16s[i] = d1; ob16[i] = d2; ob16s[i] = d3;
}

static uint64_t s = 0x12345678abcdefull;
static uint32_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)(s >> 11); }

int main(int argc, char** argv)
{
    const int n = 1 << 20;
    std::vector<float> a(n), b(n);
    std::vector<uint32_t> r(n);
    for (int i = 0; i < n; ++i) {
        uint32_t ua = rnd(), ub = rnd();
        int cls = i % 8;
        auto mk = [&](uint32_t u, int c) -> float {
            // exponent range chosen per class
            uint32_t sign = u & 0x80000000u, man = u & 0x7FFFFFu;
            int e;
            switch (c) {
            case 0: e = 127 + (int)(rnd() % 30) - 14; break;          // f16 normal range
            case 1: e = 127 - 15 - (int)(rnd() % 12); break;          // f16 subnormal / underflow
            case 2: e = 127 + 15; break;                              // near f16 max
            case 3: e = 127 + (int)(rnd() % 60) - 30; break;          // wide
            case 4: e = 1 + (int)(rnd() % 253); break;                // any finite
            case 5: e = 127 - 126 + (int)(rnd() % 4) - 1; break;      // f32 subnormal edge (bf16)
            case 6: e = 127 + 12 + (int)(rnd() % 4); break;           // large raw values
            default: e = 127 + (int)(rnd() % 10) - 5; break;
            }
            if (e < 0) e = 0;
            if (e > 254) e = 254;
            return __builtin_bit_cast(float, sign | ((uint32_t)e << 23) | man);
        };
        a[i] = mk(ua, cls);
        b[i] = mk(ub, (cls + 3) % 8);
        r[i] = rnd();
    }
    // structured: single-bit rbits with all-ones discarded fractions
    for (int k = 0; k < 32; ++k) {
        int i = k;
        a[i] = __builtin_bit_cast(float, 0x3F801FFFu);   // 1 + 0x1FFF ulp (f16 discard = 0x1FFF)
        b[i] = __builtin_bit_cast(float, 0x3F801FFFu);
        r[i] = 1u << k;
        int j = 32 + k;
        a[j] = __builtin_bit_cast(float, 0x3F80FFFFu);   // bf16 discard = 0xFFFF
        b[j] = __builtin_bit_cast(float, 0x3F80FFFFu);
        r[j] = 1u << k;
        int m = 64 + k;
        a[m] = 1.0f; b[m] = 1.0f; r[m] = 1u << k;
        // special values
    }
    float spec[] = {0.0f, -0.0f, __builtin_inff(), -__builtin_inff(), __builtin_nanf(""), 65504.0f, 65520.0f, 65536.0f,
                    1e30f, -1e30f, 5.96e-8f, 2.98e-8f, 1e-45f};
    for (int k = 0; k < 13; ++k) for (int t = 0; t < 4; ++t) {
        int i = 96 + 4 * k + t;
        a[i] = spec[k]; b[i] = -spec[k]; r[i] = t == 0 ? 0u : t == 1 ? 0xFFFFFFFFu : rnd();
    }
    float *da, *db; uint32_t *dr, *o[4];
    cudaMalloc(&da, n * 4); cudaMalloc(&db, n * 4); cudaMalloc(&dr, n * 4);
    for (int q = 0; q < 4; ++q) cudaMalloc(&o[q], n * 4);
    cudaMemcpy(da, a.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(db, b.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dr, r.data(), n * 4, cudaMemcpyHostToDevice);
    k<<<(n + 255) / 256, 256>>>(da, db, dr, o[0], o[1], o[2], o[3], n);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { fprintf(stderr, "cuda: %s\n", cudaGetErrorString(e)); return 1; }
    std::vector<uint32_t> h(4 * (size_t)n);
    for (int q = 0; q < 4; ++q) cudaMemcpy(h.data() + (size_t)q * n, o[q], n * 4, cudaMemcpyDeviceToHost);
    FILE* f = fopen(argc > 1 ? argv[1] : "cvt_rs_probe.bin", "wb");
    fwrite(&n, 4, 1, f);
    fwrite(a.data(), 4, n, f); fwrite(b.data(), 4, n, f); fwrite(r.data(), 4, n, f);
    fwrite(h.data(), 4, 4 * (size_t)n, f);
    fclose(f);
    printf("probe ok n=%d\n", n);
    return 0;
}
