// The reference's texel filters as device operations on one tile (crates/lightbaker/src/filter.rs:
// smooth :20-53, fill :58-94, sun_field :106-141): arrays in device memory, w x h texels row by row,
// `channels` floats a texel interleaved, enqueued on the handle's stream. Sums run in the reference's
// order; the Gaussian weights are computed on the host as the reference computes them, so results
// equal the host's (and the oracle's) bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "lb_device.cuh"
#include "lb_runtime.h"

namespace lbd {

constexpr int MAX_R = 8;  // smoothing radius a launch's weight table holds
struct Weights {
    float w[(2 * MAX_R + 1) * (2 * MAX_R + 1)];
};

__device__ __forceinline__ bool same_surface(const uint32_t *chart, const float *normal, uint32_t i, uint32_t j) {
    if (chart[i] != chart[j]) return false;
    const float *a = normal + 3 * size_t(i), *b = normal + 3 * size_t(j);
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] >= 0.9f;
}

template <int N>
__global__ void k_tile_smooth(uint32_t w, uint32_t h, const uint32_t *chart, const float *normal, const float *v,
                              const uint8_t *valid, int r, Weights W, float *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    int x = int(i % w), y = int(i / w);
    float sum[N], wsum = 0.0f;
    for (int c = 0; c < N; c++) sum[c] = 0.0f;
    if (!valid[i] || r == 0) {
        for (int c = 0; c < N; c++) out[size_t(i) * N + c] = v[size_t(i) * N + c];
        return;
    }
    for (int yy = y > r ? y - r : 0; yy < min(y + r + 1, int(h)); yy++)
        for (int xx = x > r ? x - r : 0; xx < min(x + r + 1, int(w)); xx++) {
            uint32_t j = uint32_t(yy) * w + uint32_t(xx);
            if (!valid[j] || !same_surface(chart, normal, i, j)) continue;
            float k = W.w[(yy - y + r) * (2 * r + 1) + (xx - x + r)];
            for (int c = 0; c < N; c++) sum[c] += v[size_t(j) * N + c] * k;
            wsum += k;
        }
    for (int c = 0; c < N; c++) out[size_t(i) * N + c] = sum[c] / wsum;
}

// one ring: reads (was, src), writes (now, dst)
template <int N>
__global__ void k_tile_fill(uint32_t w, uint32_t h, const uint32_t *chart, const uint8_t *was, const float *src,
                            uint8_t *now, float *dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    float o[N];
    for (int c = 0; c < N; c++) o[c] = src[size_t(i) * N + c];
    uint8_t k = was[i];
    if (!k) {
        int x = int(i % w), y = int(i / w);
        uint32_t ci = chart[i];
        float own[N], any[N];
        for (int c = 0; c < N; c++) own[c] = any[c] = 0.0f;
        int no = 0, na = 0;
        for (int yy = y > 0 ? y - 1 : 0; yy < min(y + 2, int(h)); yy++)
            for (int xx = x > 0 ? x - 1 : 0; xx < min(x + 2, int(w)); xx++) {
                uint32_t j = uint32_t(yy) * w + uint32_t(xx);
                if (!was[j]) continue;
                if (ci != NONE && chart[j] == ci) {
                    for (int c = 0; c < N; c++) own[c] += src[size_t(j) * N + c];
                    no++;
                } else {
                    for (int c = 0; c < N; c++) any[c] += src[size_t(j) * N + c];
                    na++;
                }
            }
        if (no > 0) {
            for (int c = 0; c < N; c++) o[c] = own[c] / float(no);
            k = 1;
        } else if (na > 0 && ci == NONE) {
            for (int c = 0; c < N; c++) o[c] = any[c] / float(na);
            k = 1;
        }
    }
    now[i] = k;
    for (int c = 0; c < N; c++) dst[size_t(i) * N + c] = o[c];
}

__global__ void k_tile_sun_field(uint32_t w, uint32_t h, const uint32_t *chart, const float *normal,
                                 const uint32_t *hard, const uint8_t *covered, int g, float radius, float *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    float res = -1.0f;
    if (covered[i]) {
        int x = int(i % w), y = int(i / w);
        int gg = g * g, reach = int(ceilf(radius)) + 1;
        bool lit = __popc(hard[i]) * 2 >= gg;
        float best = radius, fg = float(g), half = 0.5f / fg;
        for (int yy = y > reach ? y - reach : 0; yy < min(y + reach + 1, int(h)); yy++)
            for (int xx = x > reach ? x - reach : 0; xx < min(x + reach + 1, int(w)); xx++) {
                uint32_t j = uint32_t(yy) * w + uint32_t(xx);
                if (!covered[j] || !same_surface(chart, normal, i, j)) continue;
                uint32_t other = lit ? ~hard[j] : hard[j];
                if (gg < 32) other &= (1u << gg) - 1u;
                while (other) {
                    int c = __ffs(other) - 1;
                    other &= other - 1;
                    float px = float(xx) + (float(c % g) + 0.5f) / fg - (float(x) + 0.5f);
                    float py = float(yy) + (float(c / g) + 0.5f) / fg - (float(y) + 0.5f);
                    best = fminf(best, sqrtf(px * px + py * py) - half);
                }
            }
        float d = fminf(fmaxf(best, 0.0f), radius);
        res = 0.5f + 0.5f * (lit ? d : -d) / radius;
    }
    out[i] = res;
}

template <int N>
cudaError_t fill_rings(uint32_t w, uint32_t h, const uint32_t *chart, float *v, uint8_t *valid, int rings, float *sv,
                       uint8_t *sk, cudaStream_t st) {
    uint32_t n = w * h;
    dim3 grid((n + 255) / 256);
    float *vw = v, *vn = sv;
    uint8_t *kw = valid, *kn = sk;
    for (int r = 0; r < rings; r++) {
        // cudaLaunchKernel returns this launch's own status: an error the host application left in the thread
        // before this call is neither consumed nor reported as this call's
        void *args[] = {&w, &h, (void *)&chart, &kw, &vw, &kn, &vn};
        cudaError_t e = cudaLaunchKernel((const void *)k_tile_fill<N>, grid, dim3(256), args, 0, st);
        if (e != cudaSuccess) return e;
        float *t = vw;
        vw = vn;
        vn = t;
        uint8_t *u = kw;
        kw = kn;
        kn = u;
    }
    if (vw != v) {
        cudaError_t e = cudaMemcpyAsync(v, vw, size_t(n) * N * 4, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(valid, kw, n, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace lbd

// Runs `rings` fill rings with the given scratch (n * channels floats, n bytes): shared by lb_fill and its
// fixed-scratch variant.
cudaError_t lb_fill_with_scratch(uint32_t w, uint32_t h, const uint32_t *chart, float *values, int channels,
                                 uint8_t *valid, int rings, float *sv, uint8_t *sk, cudaStream_t st) {
    switch (channels) {
    case 1: return lbd::fill_rings<1>(w, h, chart, values, valid, rings, sv, sk, st);
    case 2: return lbd::fill_rings<2>(w, h, chart, values, valid, rings, sv, sk, st);
    case 3: return lbd::fill_rings<3>(w, h, chart, values, valid, rings, sv, sk, st);
    case 4: return lbd::fill_rings<4>(w, h, chart, values, valid, rings, sv, sk, st);
    default: return cudaErrorInvalidValue;
    }
}

extern "C" {

int lb_smooth(lb_gpu *g, uint32_t w, uint32_t h, const uint32_t *chart, const float *normal, const float *values,
              int channels, const uint8_t *valid, int radius, float *out) {
    if (!g || !chart || !normal || !values || !valid || !out || channels < 1 || channels > 4 || radius < 0 ||
        radius > lbd::MAX_R || w == 0 || h == 0 || uint64_t(w) * h > 0xffffffffu) {
        lb_set_error("lb_smooth: bad arguments (channels 1..4, radius 0..8)");
        return LB_EINVAL;
    }
    lbd::Weights W;
    std::memset(&W, 0, sizeof W);
    if (radius > 0) {
        float q = float(radius) * 0.75f;
        float sigma2 = 2.0f * (q * q);
        for (int dy = -radius; dy <= radius; dy++)
            for (int dx = -radius; dx <= radius; dx++) {
                float fx = float(dx), fy = float(dy);
                W.w[(dy + radius) * (2 * radius + 1) + (dx + radius)] = std::exp(-(fx * fx + fy * fy) / sigma2);
            }
    }
    uint32_t n = w * h;
    dim3 grid((n + 255) / 256);
    switch (channels) {
    case 1: lbd::k_tile_smooth<1><<<grid, 256, 0, g->stream>>>(w, h, chart, normal, values, valid, radius, W, out); break;
    case 2: lbd::k_tile_smooth<2><<<grid, 256, 0, g->stream>>>(w, h, chart, normal, values, valid, radius, W, out); break;
    case 3: lbd::k_tile_smooth<3><<<grid, 256, 0, g->stream>>>(w, h, chart, normal, values, valid, radius, W, out); break;
    default: lbd::k_tile_smooth<4><<<grid, 256, 0, g->stream>>>(w, h, chart, normal, values, valid, radius, W, out); break;
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LB_OK : lb_cuda_fail(e, "lb_smooth");
}

int lb_fill(lb_gpu *g, uint32_t w, uint32_t h, const uint32_t *chart, float *values, int channels, uint8_t *valid,
            int rings) {
    if (!g || !chart || !values || !valid || channels < 1 || channels > 4 || rings < 0 || w == 0 || h == 0 ||
        uint64_t(w) * h > 0xffffffffu) {
        lb_set_error("lb_fill: bad arguments (channels 1..4)");
        return LB_EINVAL;
    }
    size_t n = size_t(w) * h;
    // ping-pong scratch, kept by the handle
    int rc = lb_buffer_reserve(g->scratch, n * channels * 4 + n + 256);
    if (rc != LB_OK) return rc;
    float *sv = (float *)g->scratch.ptr;
    uint8_t *sk = (uint8_t *)g->scratch.ptr + ((n * channels * 4 + 255) & ~size_t(255));
    cudaError_t e = lb_fill_with_scratch(w, h, chart, values, channels, valid, rings, sv, sk, g->stream);
    return e == cudaSuccess ? LB_OK : lb_cuda_fail(e, "lb_fill");
}

int lb_sun_field(lb_gpu *g, uint32_t w, uint32_t h, const uint32_t *chart, const float *normal, const uint32_t *hard,
                 const uint8_t *covered, uint32_t grid_side, float radius, float *out) {
    if (!g || !chart || !normal || !hard || !covered || !out || grid_side < 1 || grid_side > 5 || !(radius > 0.0f) ||
        w == 0 || h == 0 || uint64_t(w) * h > 0xffffffffu) {
        lb_set_error("lb_sun_field: bad arguments (grid side 1..5, radius > 0)");
        return LB_EINVAL;
    }
    uint32_t n = w * h;
    lbd::k_tile_sun_field<<<(n + 255) / 256, 256, 0, g->stream>>>(w, h, chart, normal, hard, covered, int(grid_side),
                                                                  radius, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? LB_OK : lb_cuda_fail(e, "lb_sun_field");
}

}  // extern "C"

// ---- lb_fill_fixed: the fill with its ping-pong copy in a fixed device array, allocating nothing ----

namespace {
constexpr uint32_t FIXED_TEXELS = 512u * 512u;  // the largest tile lb_fill_fixed takes
constexpr size_t FIXED_VALUES = size_t(FIXED_TEXELS) * 4 * sizeof(float);
}  // namespace

// The scratch every lb_fill_fixed call on a device uses: FIXED_TEXELS texels of four channels and their
// flags (4.25 MiB), held by every GPU that loads the library until the process exits.
static __device__ __align__(256) unsigned char lb_fill_scratch[FIXED_VALUES + FIXED_TEXELS];

namespace {
// The array's device address belongs to a CUDA context: each context that loads the library's module has its
// own copy of the array at its own address. Host code may not take it by name, so it is looked up with
// cudaGetSymbolAddress and cached under the context's unique id (cuCtxGetId: never reused within a process, so
// a context destroyed by cudaDeviceReset or by the application, and one created later, never share an entry).
typedef int (*ctx_get_current_fn)(void **);
typedef int (*ctx_get_id_fn)(void *, unsigned long long *);
struct FixedEntry {
    unsigned long long ctx_id;
    void *ptr;
};
std::mutex g_fixed_mutex;
FixedEntry g_fixed[64];
int g_fixed_n = 0, g_fixed_next = 0;
ctx_get_current_fn g_ctx_current = nullptr;
ctx_get_id_fn g_ctx_id = nullptr;

// The unique id of the calling thread's current context (creating the device's primary context when none is
// current, as any runtime call would). Driver entry points are taken through the runtime, so the library does
// not link libcuda.
cudaError_t current_context_id(unsigned long long *id) {
    if (!g_ctx_current || !g_ctx_id) {
        cudaDriverEntryPointQueryResult q1, q2;
        cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void **)&g_ctx_current, 12000,
                                                         cudaEnableDefault, &q1);
        if (e == cudaSuccess)
            e = cudaGetDriverEntryPointByVersion("cuCtxGetId", (void **)&g_ctx_id, 12000, cudaEnableDefault, &q2);
        if (e != cudaSuccess) return e;
        if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !g_ctx_current || !g_ctx_id) {
            g_ctx_current = nullptr;
            g_ctx_id = nullptr;
            return cudaErrorSymbolNotFound;
        }
    }
    void *ctx = nullptr;
    if (g_ctx_current(&ctx) != 0) return cudaErrorDeviceUninitialized;
    if (!ctx) {
        // no context is current yet: make the runtime bind the device's primary context (no allocation)
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaSetDevice(dev);
        if (e != cudaSuccess) return e;
        if (g_ctx_current(&ctx) != 0 || !ctx) return cudaErrorDeviceUninitialized;
    }
    return g_ctx_id(ctx, id) == 0 ? cudaSuccess : cudaErrorDeviceUninitialized;
}
}  // namespace

extern "C" int lb_fill_fixed(void *stream, uint32_t w, uint32_t h, const uint32_t *chart, float *values, int channels,
                             uint8_t *valid, int rings) {
    if (!chart || !values || !valid || channels < 1 || channels > 4 || rings < 0 || w == 0 || h == 0) {
        lb_set_error("lb_fill_fixed: bad arguments (channels 1..4)");
        return LB_EINVAL;
    }
    if (uint64_t(w) * h > FIXED_TEXELS) {
        lb_set_error("lb_fill_fixed: a tile of " + std::to_string(uint64_t(w) * h) + " texels is over the fixed scratch's " +
                     std::to_string(FIXED_TEXELS) + " (512 x 512); use lb_fill");
        return LB_ESCRATCH;
    }
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_fixed_mutex);
        unsigned long long id = 0;
        cudaError_t e = current_context_id(&id);
        if (e != cudaSuccess) return lb_cuda_fail(e, "lb_fill_fixed: current context");
        for (int k = 0; k < g_fixed_n; k++)
            if (g_fixed[k].ctx_id == id) base = g_fixed[k].ptr;
        if (!base) {
            // The first call in a context looks the address up, which may load the library's module into the
            // context: not allowed while the caller's stream is being captured into a graph.
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            e = cudaStreamIsCapturing((cudaStream_t)stream, &cs);
            if (e != cudaSuccess) return lb_cuda_fail(e, "lb_fill_fixed: cudaStreamIsCapturing");
            if (cs != cudaStreamCaptureStatusNone) {
                lb_set_error("lb_fill_fixed: the first call in a CUDA context must come before any stream capture "
                             "(it looks up the fixed scratch's address); call it once outside the capture");
                return LB_EINVAL;
            }
            e = cudaGetSymbolAddress(&base, lb_fill_scratch);
            if (e != cudaSuccess) return lb_cuda_fail(e, "lb_fill_fixed: cudaGetSymbolAddress");
            g_fixed[g_fixed_next] = {id, base};  // a ring of 64 contexts: the oldest entry goes first
            g_fixed_next = (g_fixed_next + 1) % 64;
            if (g_fixed_n < 64) g_fixed_n++;
        }
    }
    float *sv = (float *)base;
    uint8_t *sk = (uint8_t *)base + FIXED_VALUES;
    cudaError_t e = lb_fill_with_scratch(w, h, chart, values, channels, valid, rings, sv, sk, (cudaStream_t)stream);
    return e == cudaSuccess ? LB_OK : lb_cuda_fail(e, "lb_fill_fixed");
}
