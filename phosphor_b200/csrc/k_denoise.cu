// k_denoise.cu — the reference denoiser's image filters on the GPU (denoise/filters_gpu.py:9-86:
// mean_filter, median_filter, weighted_filter), behind phx_mean_filter / phx_median_filter /
// phx_weighted_filter.
//
// Input: an (H, W, 3) int32 image, as filters_gpu.py:_run_kernel passes it; output (H, W, 3)
// float32.  Every output pixel and channel reads the window [clamp(x-k), clamp(x+k)] x
// [clamp(y-k), clamp(y+k)] — clamped to the image, so border windows shrink — and sums in the
// reference's order (xx outer, yy inner) with one rounding per float operation (the library is
// built without contraction), so the results are the reference kernels' bits.
//
// Layout: one thread per pixel in 32 x 8 blocks; for k <= TILE_K the block first stages its
// (32 + 2k) x (8 + 2k) window of the image in shared memory with coalesced loads (each image
// pixel is then read from HBM once per block instead of (2k+1)^2 times through L1), and the
// weights too.  Larger windows read the image through the read-only cache.
#include "kernels.hpp"

#include <type_traits>

namespace phx {

namespace {

constexpr int BX = 32, BY = 8;
constexpr int TILE_K = 8; // largest window radius staged in shared memory (48 x 24 x 3 ints)
constexpr int TILE_W = BX + 2 * TILE_K, TILE_H = BY + 2 * TILE_K;

enum : int { F_MEAN = 0, F_MEDIAN = 1, F_WEIGHTED = 2 };

// Ascending bitonic sorting network over N (a power of two) values in registers: every index is a
// compile-time constant once unrolled, so nothing goes to local memory.
template <int N> __device__ void bitonic_sort(int (&a)[N]) {
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < N; i++) {
                const int l = i ^ j;
                if (l > i) {
                    const int x = a[i], y = a[l];
                    const bool up = (i & k) == 0;
                    a[i] = up ? min(x, y) : max(x, y);
                    a[l] = up ? max(x, y) : min(x, y);
                }
            }
}

// The median of the window's n values (the rest of `v` is INT_MAX padding, sorted last), as
// median_filter's insertion sort then takes it (filters_gpu.py:57-62): the mean of the two middle
// values, (a + b) / 2.0f with an integer sum, for an even n, else the middle value.
template <int N> __device__ float median_of(int (&v)[N], int n) {
    bitonic_sort(v);
    const int rlo = (n - 1) / 2, rhi = n / 2;
    int lo = 0, hi = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        lo = i == rlo ? v[i] : lo;
        hi = i == rhi ? v[i] : hi;
    }
    return (n % 2 == 0) ? (float)(lo + hi) / 2.0f : (float)hi;
}

template <int N> struct Pow2 {
    static constexpr int value = N <= 1 ? 1 : 2 * Pow2<(N + 1) / 2>::value;
};
template <> struct Pow2<1> {
    static constexpr int value = 1;
};

// MODE: F_MEAN / F_MEDIAN / F_WEIGHTED.  TILED: the block's window of the image (and the weights)
// staged in shared memory, for k <= TILE_K.  MK: the median's window radius (compile time).
// The image is staged as float for the sums (each value converted once: the same value the
// kernels' per-use (float) conversion gives) and as int for the median.  The three channels are
// summed together; each channel's additions keep the kernels' order.
template <int MODE, bool TILED, int MK>
__global__ void __launch_bounds__(BX *BY) k_filter(const int *__restrict__ in, float *__restrict__ out,
                                                   const float *__restrict__ weights, int width, int height, int k) {
    using T = typename std::conditional<MODE == F_MEDIAN, int, float>::type;
    __shared__ T tile[TILED ? TILE_H * TILE_W * 3 : 1];
    __shared__ float wsh[TILED && MODE == F_WEIGHTED ? (2 * TILE_K + 1) * (2 * TILE_K + 1) : 1];
    const int x0 = blockIdx.x * BX - k, y0 = blockIdx.y * BY - k; // tile origin in the image
    if constexpr (TILED) {
        // row by row: a tile row is 3 * (BX + 2k) consecutive ints of one image row (coalesced)
        const int gxa = max(x0, 0), gxb = min(x0 + BX + 2 * k, width); // image columns [gxa, gxb)
        const int rowlen = 3 * (gxb - gxa), skip = 3 * (gxa - x0);
        for (int ty = threadIdx.y; ty < BY + 2 * k; ty += BY) {
            const int gy = y0 + ty;
            if (gy < 0 || gy >= height) // rows outside the image are never read
                continue;
            const int *src = in + ((size_t)gy * width + gxa) * 3;
            T *dst = tile + ty * TILE_W * 3 + skip;
            for (int i = threadIdx.x; i < rowlen; i += BX)
                dst[i] = (T)__ldg(&src[i]);
        }
        if constexpr (MODE == F_WEIGHTED) {
            const int nw = (2 * k + 1) * (2 * k + 1);
            for (int i = threadIdx.y * BX + threadIdx.x; i < nw; i += BX * BY)
                wsh[i] = __ldg(&weights[i]);
        }
        __syncthreads();
    }
    const int x = blockIdx.x * BX + threadIdx.x, y = blockIdx.y * BY + threadIdx.y;
    if (x >= width || y >= height)
        return;
    // channel c of pixel (xx, yy), which lies in this pixel's clamped window
    auto px = [&](int xx, int yy, int c) -> T {
        if constexpr (TILED)
            return tile[((yy - y0) * TILE_W + (xx - x0)) * 3 + c];
        else
            return (T)__ldg(&in[((size_t)yy * width + xx) * 3 + c]);
    };
    const int xa = max(x - k, 0), xb = min(x + k, width - 1);
    const int ya = max(y - k, 0), yb = min(y + k, height - 1);
    float r[3];
    if constexpr (MODE == F_MEAN) { // filters_gpu.py:9-27
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
        for (int xx = xa; xx <= xb; xx++)
            for (int yy = ya; yy <= yb; yy++) {
                s0 += px(xx, yy, 0);
                s1 += px(xx, yy, 1);
                s2 += px(xx, yy, 2);
            }
        const float n = (float)((xb - xa + 1) * (yb - ya + 1)); // the kernel's count i
        r[0] = s0 / n;
        r[1] = s1 / n;
        r[2] = s2 / n;
    } else if constexpr (MODE == F_MEDIAN) { // filters_gpu.py:29-67 (k <= 2)
        constexpr int W = (2 * MK + 1) * (2 * MK + 1), N = Pow2<W>::value;
        const int n = (xb - xa + 1) * (yb - ya + 1);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            int v[N];
#pragma unroll
            for (int dx = -MK; dx <= MK; dx++)
#pragma unroll
                for (int dy = -MK; dy <= MK; dy++) {
                    const int xx = x + dx, yy = y + dy;
                    const bool ok = xx >= xa && xx <= xb && yy >= ya && yy <= yb;
                    const int val = px(min(max(xx, xa), xb), min(max(yy, ya), yb), c); // always in the window
                    v[(dx + MK) * (2 * MK + 1) + (dy + MK)] = ok ? val : 0x7fffffff;
                }
#pragma unroll
            for (int i = W; i < N; i++)
                v[i] = 0x7fffffff;
            r[c] = median_of(v, n);
        }
    } else { // filters_gpu.py:69-86
        const int ks = 2 * k + 1;
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
        for (int xx = xa; xx <= xb; xx++)
            for (int yy = ya; yy <= yb; yy++) {
                const int widx = (yy - y + k) * ks + (xx - x + k);
                float wv;
                if constexpr (TILED)
                    wv = wsh[widx];
                else
                    wv = __ldg(&weights[widx]);
                s0 += px(xx, yy, 0) * wv;
                s1 += px(xx, yy, 1) * wv;
                s2 += px(xx, yy, 2) * wv;
            }
        r[0] = s0;
        r[1] = s1;
        r[2] = s2;
    }
    float *o = out + ((size_t)y * width + x) * 3;
    o[0] = r[0];
    o[1] = r[1];
    o[2] = r[2];
}

template <int MODE, int MK> void launch_mode(const int *in, float *out, const float *w, int width, int height, int k,
                                             cudaStream_t st) {
    const dim3 block(BX, BY), grid((width + BX - 1) / BX, (height + BY - 1) / BY);
    if (k <= TILE_K)
        k_filter<MODE, true, MK><<<grid, block, 0, st>>>(in, out, w, width, height, k);
    else
        k_filter<MODE, false, MK><<<grid, block, 0, st>>>(in, out, w, width, height, k);
}

} // namespace

// Runs one filter on host arrays: copies in, one kernel, copies out.  Returns 0, or 1 (invalid
// argument) / 3 (CUDA error) with `msg` set; *kernel_ms (if given) is the kernel's CUDA-event time.
int denoise_filter(int mode, const int32_t *in, float *out, const float *weights, uint32_t width, uint32_t height,
                   uint32_t k, float *kernel_ms, std::string &msg) {
    if (!in || !out || (mode == F_WEIGHTED && !weights)) {
        msg = "null buffer";
        return 1;
    }
    if (width == 0 || height == 0 || (uint64_t)width * height * 3 > 0x7fffffffull) {
        msg = "image size must be 1..2^31/3 pixels";
        return 1;
    }
    if (mode == F_MEDIAN && k > 2) {
        msg = "median filter k is > 3"; // filters_gpu.py:138-139 raises for k > 2
        return 1;
    }
    if (k > 32) {
        msg = "window radius k must be <= 32";
        return 1;
    }
    const size_t n = (size_t)width * height * 3, nw = (size_t)(2 * k + 1) * (2 * k + 1);
    cudaStream_t st = nullptr;
    int *d_in = nullptr;
    float *d_out = nullptr, *d_w = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    auto ok = [&]() { return err == cudaSuccess; };
    if (ok())
        err = cudaMallocAsync((void **)&d_in, n * sizeof(int), st);
    if (ok())
        err = cudaMallocAsync((void **)&d_out, n * sizeof(float), st);
    if (ok() && mode == F_WEIGHTED)
        err = cudaMallocAsync((void **)&d_w, nw * sizeof(float), st);
    if (ok())
        err = cudaMemcpyAsync(d_in, in, n * sizeof(int), cudaMemcpyHostToDevice, st);
    if (ok() && d_w)
        err = cudaMemcpyAsync(d_w, weights, nw * sizeof(float), cudaMemcpyHostToDevice, st);
    if (ok() && kernel_ms) {
        err = cudaEventCreate(&e0);
        if (ok())
            err = cudaEventCreate(&e1);
        if (ok())
            err = cudaEventRecord(e0, st);
    }
    if (ok()) {
        const int w = (int)width, h = (int)height, kk = (int)k;
        if (mode == F_MEAN)
            launch_mode<F_MEAN, 0>(d_in, d_out, nullptr, w, h, kk, st);
        else if (mode == F_WEIGHTED)
            launch_mode<F_WEIGHTED, 0>(d_in, d_out, d_w, w, h, kk, st);
        else if (k == 0)
            launch_mode<F_MEDIAN, 0>(d_in, d_out, nullptr, w, h, kk, st);
        else if (k == 1)
            launch_mode<F_MEDIAN, 1>(d_in, d_out, nullptr, w, h, kk, st);
        else
            launch_mode<F_MEDIAN, 2>(d_in, d_out, nullptr, w, h, kk, st);
        err = cudaGetLastError();
    }
    if (ok() && kernel_ms)
        err = cudaEventRecord(e1, st);
    if (ok())
        err = cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (ok())
        err = cudaStreamSynchronize(st);
    if (ok() && kernel_ms)
        err = cudaEventElapsedTime(kernel_ms, e0, e1);
    const cudaError_t first = err;
    if (st) { // release in every case; the first error is the one reported
        if (d_in)
            cudaFreeAsync(d_in, st);
        if (d_out)
            cudaFreeAsync(d_out, st);
        if (d_w)
            cudaFreeAsync(d_w, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (e0)
        cudaEventDestroy(e0);
    if (e1)
        cudaEventDestroy(e1);
    if (first != cudaSuccess) {
        msg = std::string("CUDA error: ") + cudaGetErrorString(first);
        return 3;
    }
    return 0;
}

} // namespace phx
