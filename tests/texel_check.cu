// Checks tex_texel (mcsart_b200/csrc/common.cuh) against the hardware: a
// linear-filtered float texture, configured as the reference backprojector's
// (src/cu_backprojection.cu:28-33), fetched at texel centres.  Texels of every
// sign and magnitude class (denormals, the smallest normals, normals, zeros);
// prints the number of fetches that differ from tex_texel of the texel.
#include <cstdio>
#include <cstring>

#include "common.cuh"

using namespace mcsart;

__global__ void fetch(cudaTextureObject_t t, const float *texels, unsigned *bad, int na, int nb) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
    if (a >= na || b >= nb) return;
    const float got = tex3D<float>(t, a + 0.5f, b + 0.5f, 0.5f);
    if (__float_as_uint(got) != __float_as_uint(tex_texel(texels[a + b * na]))) atomicAdd(bad, 1u);
}

int main() {
    const int na = 1024, nb = 64, n = na * nb;
    static unsigned h[n];
    unsigned s = 12345u;
    for (int i = 0; i < n; i++) {
        s ^= s << 13; s ^= s >> 17; s ^= s << 5;
        const unsigned sign = (s & 1u) << 31;
        switch (i % 5) {
            case 0: h[i] = sign | (s >> 9); break;                        // denormal or zero
            case 1: h[i] = sign | 0x00800000u | (s >> 9); break;          // smallest normals
            case 2: h[i] = sign | ((1u + (s % 253u)) << 23) | (s >> 9); break;  // normals
            case 3: h[i] = sign; break;                                   // +-0
            default: h[i] = sign | 1u; break;                             // smallest denormal
        }
    }
    float *d = nullptr;
    unsigned *bad = nullptr, hb = 0;
    if (cudaMalloc(&d, sizeof(h)) != cudaSuccess || cudaMalloc(&bad, sizeof(unsigned)) != cudaSuccess)
        return 2;
    cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice);
    cudaMemset(bad, 0, sizeof(unsigned));
    const cudaChannelFormatDesc cd = cudaCreateChannelDesc(32, 0, 0, 0, cudaChannelFormatKindFloat);
    cudaArray_t arr;
    if (cudaMalloc3DArray(&arr, &cd, make_cudaExtent(na, nb, 1)) != cudaSuccess) return 2;
    cudaMemcpy3DParms p;
    memset(&p, 0, sizeof(p));
    p.srcPtr = make_cudaPitchedPtr(h, na * sizeof(float), na, nb);
    p.dstArray = arr;
    p.extent = make_cudaExtent(na, nb, 1);
    p.kind = cudaMemcpyHostToDevice;
    if (cudaMemcpy3D(&p) != cudaSuccess) return 2;
    cudaResourceDesc rd;
    memset(&rd, 0, sizeof(rd));
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) return 2;
    fetch<<<dim3(na / 256, nb), 256>>>(t, d, bad, na, nb);
    if (cudaDeviceSynchronize() != cudaSuccess) return 3;
    cudaMemcpy(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost);
    printf("%u\n", hb);
    cudaDestroyTextureObject(t);
    cudaFreeArray(arr);
    cudaFree(d);
    cudaFree(bad);
    return 0;
}
