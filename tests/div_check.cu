// Checks the engine's branch-free division (mk_recip / mk_div in
// mcsart_b200/csrc/common.cuh) bit for bit against the compiler's correctly
// rounded reciprocal and division: every significand of the divisor for
// exponents -20 .. 19, and random quotients (projector-weight operands and
// operands over 2^-20 .. 2^20); and the magic-number conversions (mk_floor,
// mk_floor_i, mk_i2f) against floorf and int-to-float for
// every float of magnitude below 2^22 and every int in [-2^22, 2^22).  Prints
// five mismatch counts.
#include <cstdio>

#include "common.cuh"

using namespace mcsart;

__global__ void check_exhaustive(unsigned long long *bad, int e0) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= (1u << 23)) return;
    const int e = e0 + (int)blockIdx.y;
    const float b = __uint_as_float(((uint32_t)(e + 127) << 23) | m);
    const float y = mk_recip(b);
    if (__float_as_uint(y) != __float_as_uint(__frcp_rn(b))) atomicAdd(&bad[0], 1ull);
    uint32_t h = m * 2654435761u + (uint32_t)e * 40503u + 1u;
    for (int i = 0; i < 4; i++) {
        h ^= h << 13; h ^= h >> 17; h ^= h << 5;
        const float a = __uint_as_float(((uint32_t)(124 + (h & 7)) << 23) | (h >> 9)) *
                        ((h & 256) ? -1.0f : 1.0f);
        if (__float_as_uint(mk_div(a, b, y)) != __float_as_uint(__fdiv_rn(a, b)))
            atomicAdd(&bad[1], 1ull);
    }
}

__global__ void check_random(unsigned long long *bad, uint32_t seed, int n_per) {
    uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) * 747796405u + seed * 2891336453u + 1u;
    for (int i = 0; i < n_per; i++) {
        h ^= h << 13; h ^= h >> 17; h ^= h << 5; const uint32_t r1 = h;
        h ^= h << 13; h ^= h >> 17; h ^= h << 5; const uint32_t r2 = h;
        h ^= h << 13; h ^= h >> 17; h ^= h << 5; const uint32_t r3 = h;
        // a footprint weight: overlap of [fz, fz+1] with [lo, hi] over hi - lo
        const float base = ((float)(r1 >> 8) * (1.0f / 16777216.0f) - 0.5f) * 600.0f;
        const float lo = base + (float)(r2 >> 8) * (1.0f / 16777216.0f) * 3.0f;
        const float hi = lo + (float)(r3 >> 8) * (1.0f / 16777216.0f) * 4.0f + 1e-3f;
        const float fz = floorf(lo) + (float)(r2 & 1);
        const float a = __fsub_rn(fminf(__fadd_rn(fz, 1.0f), hi), fmaxf(fz, lo));
        const float b = __fsub_rn(hi, lo);
        // both signs of the numerator (-0 is outside the accepted range)
        if (mk_den_ok(b)) {
            const float y = mk_recip(b);
            if (mk_num_ok(a) && __float_as_uint(mk_div(a, b, y)) != __float_as_uint(__fdiv_rn(a, b)))
                atomicAdd(&bad[2], 1ull);
            if (mk_num_ok(-a) &&
                __float_as_uint(mk_div(-a, b, y)) != __float_as_uint(__fdiv_rn(-a, b)))
                atomicAdd(&bad[2], 1ull);
        }
        const float a2 = __uint_as_float(((uint32_t)(107 + (r1 % 40)) << 23) | (r2 >> 9)) *
                         ((r3 & 1) ? -1.0f : 1.0f);
        const float b2 = __uint_as_float(((uint32_t)(107 + (r3 % 40)) << 23) | (r1 >> 9));
        if (__float_as_uint(mk_div(a2, b2, mk_recip(b2))) != __float_as_uint(__fdiv_rn(a2, b2)))
            atomicAdd(&bad[3], 1ull);
    }
}

// blockIdx.y = sign * 256 + biased exponent (0 .. 148: |x| < 2^22)
__global__ void check_conversions(unsigned long long *bad) {
    const uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= (1u << 23)) return;
    const uint32_t e = blockIdx.y & 255u, s = blockIdx.y >> 8;
    const float x = __uint_as_float((s << 31) | (e << 23) | m);
    if (!(fabsf(x) < MK_MAGIC_RANGE)) return;
    float fl;
    const int i = mk_floor(x, fl);
    const float rf = floorf(x);
    int n = 0;
    n += i != (int)rf;
    n += mk_floor_i(x) != (int)rf;
    n += __float_as_uint(fl) != __float_as_uint((float)(int)rf);  // a zero floor is +0
    if (e == 0) {  // every int of [-2^22, 2^22) once, from the e = 0 blocks
        const int k = (int)m - (s ? (1 << 23) : 0);  // [-2^23, 2^23)
        if (k >= -(1 << 22) && k < (1 << 22))
            n += __float_as_uint(mk_i2f(k)) != __float_as_uint((float)k);
    }
    if (n) atomicAdd(&bad[4], (unsigned long long)n);
}

int main() {
    unsigned long long *bad = nullptr, h[5] = {0, 0, 0, 0, 0};
    if (cudaMalloc(&bad, sizeof(h)) != cudaSuccess) return 2;
    cudaMemset(bad, 0, sizeof(h));
    check_exhaustive<<<dim3((1u << 23) / 256, 40), 256>>>(bad, -20);
    for (int s = 0; s < 2; s++) check_random<<<148 * 16, 256>>>(bad, 77u + s, 1024);
    check_conversions<<<dim3((1u << 23) / 256, 512), 256>>>(bad);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    cudaMemcpy(h, bad, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(bad);
    printf("%llu %llu %llu %llu %llu\n", h[0], h[1], h[2], h[3], h[4]);
    return 0;
}
