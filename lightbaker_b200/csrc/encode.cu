// The bake's output encodings on the device (crates/lightbaker/src/encode.rs:7-70, output.rs:97-101,
// :118-121, :162-181): BC5 blocks of the direct atlas, RGB9E5 words of the indirect atlas and the
// volume's 16 bytes a probe, written straight from the atlases the composite leaves in device memory, so
// a bake's file needs only its compression (zstd, deflate) on the host. Every value equals the host
// encoder's (csrc/host/encode.cpp, output.cpp) bit for bit:
// - quantisation to bytes is (clamp(v, 0, 1) * 255) rounded half away from zero (roundf), as Rust's round;
// - BC4 palettes are float sevenths compared with strict < in index order (the first nearest wins);
// - RGB9E5's exponent is floor(log2 m) as the C library's correctly rounded log2f gives it: the float
//   nearest log2(m), which for the few m just below a power of two is that power's exponent. The double
//   log2 rounded to float decides it the same way for every positive float below 65408 (an exhaustive
//   CPU check of all 1.2e9 of them); powers of two, divisions by them and floor are exact.
#include <cuda_runtime.h>

#include <cstdint>

#include "lb_runtime.h"

namespace lbd {

__device__ __forceinline__ uint8_t qbyte(float v) { return uint8_t(roundf(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f)); }

// encode.rs:7-35 on 16 values; writes 8 bytes
__device__ __forceinline__ void bc4(const uint8_t v[16], uint8_t *out) {
    uint8_t hi = v[0], lo = v[0];
    for (int k = 1; k < 16; k++) {
        hi = v[k] > hi ? v[k] : hi;
        lo = v[k] < lo ? v[k] : lo;
    }
    uint64_t bits = 0;
    if (hi != lo) {
        float pal[8];
        pal[0] = float(hi);
        pal[1] = float(lo);
        for (int i = 2; i < 8; i++) pal[i] = (float(8 - i) * float(hi) + float(i - 1) * float(lo)) / 7.0f;
        for (int k = 0; k < 16; k++) {
            float x = float(v[k]);
            int best = 0;
            for (int i = 1; i < 8; i++)
                if (fabsf(pal[i] - x) < fabsf(pal[best] - x)) best = i;
            bits |= uint64_t(best) << (3 * k);
        }
    }
    out[0] = hi;
    out[1] = lo;
    for (int b = 0; b < 6; b++) out[2 + b] = uint8_t(bits >> (8 * b));
}

// encode.rs:37-51: a thread a 4 x 4 block and channel; block (bx, by) at ((by * w/4) + bx) * 16, channel c at + 8c
__global__ void k_bc5(const float2 *direct, uint32_t w, uint32_t h, uint8_t *out) {
    uint32_t bw = w / 4, nb = bw * (h / 4);
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * nb) return;
    uint32_t b = t >> 1, c = t & 1u;
    uint32_t bx = (b % bw) * 4, by = (b / bw) * 4;
    uint8_t v[16];
    for (int k = 0; k < 16; k++) {
        float2 d = direct[size_t(by + k / 4) * w + bx + k % 4];
        v[k] = qbyte(c ? d.y : d.x);
    }
    uint8_t blk[8];
    bc4(v, blk);
    uint2 word;
    word.x = uint32_t(blk[0]) | uint32_t(blk[1]) << 8 | uint32_t(blk[2]) << 16 | uint32_t(blk[3]) << 24;
    word.y = uint32_t(blk[4]) | uint32_t(blk[5]) << 8 | uint32_t(blk[6]) << 16 | uint32_t(blk[7]) << 24;
    reinterpret_cast<uint2 *>(out)[size_t(b) * 2 + c] = word;
}

// encode.rs:53-70
__device__ __forceinline__ uint32_t rgb9e5(float r, float g, float b) {
    const float MAX = 65408.0f;
    r = fminf(fmaxf(r, 0.0f), MAX);
    g = fminf(fmaxf(g, 0.0f), MAX);
    b = fminf(fmaxf(b, 0.0f), MAX);
    float m = fmaxf(fmaxf(r, g), b);
    if (!(m > 0.0f)) return 0u;
    int e = max(int(floorf(__double2float_rn(log2(double(m))))), -16) + 1 + 15;
    float scale = ldexpf(1.0f, e - 15 - 9);
    if (uint32_t(floorf(m / scale + 0.5f)) == 512u) {
        e += 1;
        scale *= 2.0f;
    }
    auto q = [&](float v) { return min(uint32_t(floorf(v / scale + 0.5f)), 511u); };
    return q(r) | (q(g) << 9) | (q(b) << 18) | (uint32_t(e) << 27);
}

__global__ void k_rgb9e5(const float4 *v, uint32_t n, uint32_t *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 c = v[i];
    out[i] = rgb9e5(c.x, c.y, c.z);
}

// output.rs:118: the largest L0 colour of any probe, at least 1e-6 (max is exact in any order; the
// values are >= 0 after the max with 1e-6, so their bit patterns order as the floats do)
__global__ void k_volume_scale(const float4 *probes, uint32_t n, unsigned int *scale_bits) {
    float m = 1e-6f;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        float4 p = probes[size_t(k) * 4];
        m = fmaxf(m, fmaxf(fmaxf(p.x, p.y), p.z));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(scale_bits, __float_as_uint(m));
}

// output.rs:162-181: a thread a probe, 16 bytes
__global__ void k_volume_bytes(const float4 *probes, uint32_t n, const unsigned int *scale_bits, uint8_t *out) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float SQRT3 = 1.7320508f;
    float scale = __uint_as_float(*scale_bits);
    float4 p0 = probes[size_t(k) * 4];
    float l0[3] = {p0.x, p0.y, p0.z};
    uint8_t b[16];
    for (int c = 0; c < 3; c++) b[c] = qbyte(sqrtf(fmaxf(l0[c], 0.0f) / scale));
    b[3] = qbyte(p0.w);
    for (int axis = 1; axis < 4; axis++) {
        float4 pa = probes[size_t(k) * 4 + axis];
        float l1[3] = {pa.x, pa.y, pa.z};
        for (int c = 0; c < 3; c++) {
            float r = l0[c] > 1e-6f ? l1[c] / (l0[c] * SQRT3) : 0.0f;
            b[4 + (axis - 1) * 3 + c] = qbyte(r * 0.5f + 0.5f);
        }
    }
    b[13] = b[14] = b[15] = 0;
    uint4 word;
    word.x = uint32_t(b[0]) | uint32_t(b[1]) << 8 | uint32_t(b[2]) << 16 | uint32_t(b[3]) << 24;
    word.y = uint32_t(b[4]) | uint32_t(b[5]) << 8 | uint32_t(b[6]) << 16 | uint32_t(b[7]) << 24;
    word.z = uint32_t(b[8]) | uint32_t(b[9]) << 8 | uint32_t(b[10]) << 16 | uint32_t(b[11]) << 24;
    word.w = uint32_t(b[12]);
    reinterpret_cast<uint4 *>(out)[k] = word;
}

}  // namespace lbd

cudaError_t lb_encode_bc5(const float2 *direct, uint32_t w, uint32_t h, uint8_t *out, cudaStream_t st) {
    if (w % 4 || h % 4) return cudaErrorInvalidValue;
    uint32_t threads = 2 * (w / 4) * (h / 4);
    if (!threads) return cudaSuccess;
    lbd::k_bc5<<<(threads + 255) / 256, 256, 0, st>>>(direct, w, h, out);
    return cudaPeekAtLastError();
}

cudaError_t lb_encode_rgb9e5(const float4 *v, uint32_t n, uint32_t *out, cudaStream_t st) {
    if (!n) return cudaSuccess;
    lbd::k_rgb9e5<<<(n + 255) / 256, 256, 0, st>>>(v, n, out);
    return cudaPeekAtLastError();
}

cudaError_t lb_encode_volume(const float4 *probes, uint32_t n, unsigned int *scale_bits, uint8_t *out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(scale_bits, 0, 4, st);
    if (e != cudaSuccess) return e;
    uint32_t blocks = (n + 255) / 256;
    lbd::k_volume_scale<<<blocks < 1 ? 1 : (blocks > 1184 ? 1184 : blocks), 256, 0, st>>>(probes, n, scale_bits);
    if ((e = cudaPeekAtLastError()) != cudaSuccess || !n) return e;
    lbd::k_volume_bytes<<<blocks, 256, 0, st>>>(probes, n, scale_bits, out);
    return cudaPeekAtLastError();
}

extern "C" int lb_rgb9e5_device(lb_gpu *g, const float *rgba, size_t n, uint32_t *out) {
    if (!g || (n && (!rgba || !out)) || n > 0xffffffffu) {
        lb_set_error("lb_rgb9e5_device: bad arguments");
        return LB_EINVAL;
    }
    cudaError_t e = lb_encode_rgb9e5((const float4 *)rgba, uint32_t(n), out, g->stream);
    return e == cudaSuccess ? LB_OK : lb_cuda_fail(e, "lb_rgb9e5_device");
}
