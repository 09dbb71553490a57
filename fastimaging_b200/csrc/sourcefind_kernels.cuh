// Device kernels of the source finder (src/stp/sourcefind/sourcefind.cpp:22-671,
// src/stp/common/matrix_math.cpp:20-499, src/stp/common/ccl.h:19-773).
#pragma once

#include "common.cuh"

namespace stpgpu {

constexpr int SF_THREADS = 256;
// Resident blocks per SM that the streaming statistics passes are built for
// (<= 64 registers a thread: room for several wide loads in flight per
// thread) and launched with: one wave of 148 * 4 blocks.
constexpr int SF_STREAM_BLOCKS = 4;
constexpr int BINS_N = 1000; // binapprox / binmedian bin count (matrix_math.cpp:54,339)
constexpr uint32_t UF_MAX_STEPS = 1u << 26; // bound on union-find loops

template <typename T>
__device__ __forceinline__ double ld(const T* p, int64_t i)
{
    return double(p[i]);
}

// Four consecutive samples x[4g .. 4g+3] (x 16-byte aligned).
template <typename T>
__device__ __forceinline__ void load4(const T* x, int64_t g, T (&v)[4])
{
    if constexpr (sizeof(T) == 4) {
        const float4 q = reinterpret_cast<const float4*>(x)[g];
        v[0] = q.x;
        v[1] = q.y;
        v[2] = q.z;
        v[3] = q.w;
    } else {
        const double2 a = reinterpret_cast<const double2*>(x)[2 * g];
        const double2 b = reinterpret_cast<const double2*>(x)[2 * g + 1];
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
}

// Grid-stride visit of x[0..n) in 16-byte loads (four floats or two pairs of
// doubles per step, when x is 16-byte aligned), then the tail; f(value) is
// called once per element (with the element's own type).  The wide loads
// keep enough bytes in flight per thread for the streaming passes over an
// image.
template <typename T, typename F>
__device__ __forceinline__ void for_each_elem(const T* x, int64_t n, F f)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t tid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    int64_t done = 0;
    if ((reinterpret_cast<uintptr_t>(x) & 15) == 0) {
        const int64_t n4 = n / 4;
        // UNR groups of four loaded before any is used: several 16-byte
        // loads in flight per thread (64 bytes single, 64 bytes double)
        constexpr int UNR = sizeof(T) == 4 ? 4 : 2;
        int64_t g = tid;
        for (; g + (UNR - 1) * stride < n4; g += UNR * stride) {
            T a[UNR][4];
#pragma unroll
            for (int u = 0; u < UNR; u++)
                load4(x, g + u * stride, a[u]);
#pragma unroll
            for (int u = 0; u < UNR; u++)
#pragma unroll
                for (int k = 0; k < 4; k++)
                    f(a[u][k]);
        }
        for (; g < n4; g += stride) {
            T a[4];
            load4(x, g, a);
#pragma unroll
            for (int k = 0; k < 4; k++)
                f(a[k]);
        }
        done = n4 * 4;
    }
    for (int64_t i = done + tid; i < n; i += stride)
        f(x[i]);
}

// order-preserving 64-bit key of a double (non-NaN)
__device__ __forceinline__ unsigned long long okey(double v)
{
    unsigned long long u = __double_as_longlong(v);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_inv(unsigned long long k)
{
    unsigned long long u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double(u);
}

// x86 int(double) conversion (cvttsd2si): truncation, INT_MIN when out of range / NaN.
__device__ __forceinline__ int int_trunc_x86(double t)
{
    if (!(t > -2147483649.0 && t < 2147483648.0))
        return INT32_MIN;
    return int(t);
}

// -------------------------------------------------- deterministic FP64 reductions

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <int NV, int BT = SF_THREADS>
__device__ __forceinline__ void block_sums(double (&v)[NV], double* out_part)
{
    __shared__ double s[NV][BT / 32];
    for (int q = 0; q < NV; q++) {
        double w = warp_sum(v[q]);
        if ((threadIdx.x & 31) == 0)
            s[q][threadIdx.x >> 5] = w;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0.0;
        for (int k = 0; k < BT / 32; k++)
            t += s[threadIdx.x][k];
        out_part[threadIdx.x] = t;
    }
}

// Exclusive scan of v over the block (BT threads); *total = the sum.
// Callers pack up to three 16-bit counts into v.
template <int BT = SF_THREADS>
__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long v, unsigned long long* total)
{
    __shared__ unsigned long long ws[BT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        ws[warp] = x;
    __syncthreads();
    unsigned long long before = 0, all = 0;
#pragma unroll
    for (int w = 0; w < BT / 32; w++) {
        const unsigned long long t = ws[w];
        if (w < warp)
            before += t;
        all += t;
    }
    *total = all;
    __syncthreads();
    return before + x - v;
}

// -------------------------------------------------- statistics on the device
//
// The statistics of the image and the thresholds derived from them stay on
// the device from the first pass to the labeller, so the host waits only
// once, for the label counts.  A pass ends with its last block (the last to
// take a ticket) reducing every block's partials in a fixed order, so the
// results do not depend on block scheduling.

struct SfStats {
    double mean, sigma, median, rms;
    double thr[4]; // analysis +, analysis -, detection +, detection -
    unsigned long long kpos, kneg; // order keys of the detection thresholds
    unsigned int fpos, fneg; // single-precision keys of the detection thresholds rounded onto the float grid
    unsigned int need_exact; // the binned median does not apply: the exact path must run
    unsigned int stats_err; // the fused statistics kernel gave up at a grid barrier: the pass kernels must run
};

// True in exactly one block, the last to finish the pass; every other
// block's writes before the call are visible to it (the barrier, then one
// fenced ticket per block, as in a grid-wide barrier).  Resets the ticket
// for the next pass.
__device__ __forceinline__ bool last_block(unsigned int* ticket)
{
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        last = t == gridDim.x - 1;
        if (last) {
            *ticket = 0;
            __threadfence();
        }
    }
    __syncthreads();
    return last;
}

// Sum NV-wide partials of nb blocks in a fixed order (one block of BT
// threads: strided sums, warp trees, warps in order); the result is valid in
// every thread.
template <int NV, int BT = SF_THREADS>
__device__ __forceinline__ void reduce_parts(const double* part, int nb, double (&out)[NV])
{
    __shared__ double s[NV][BT / 32];
    double t[NV];
    for (int q = 0; q < NV; q++)
        t[q] = 0.0;
    // all of a thread's loads in flight together (one L2 round trip per BT
    // blocks), the same order of addition per quantity
#pragma unroll 4
    for (int k = threadIdx.x; k < nb; k += BT)
        for (int q = 0; q < NV; q++)
            t[q] += __ldcg(part + NV * k + q);
    for (int q = 0; q < NV; q++) {
        const double w = warp_sum(t[q]);
        if ((threadIdx.x & 31) == 0)
            s[q][threadIdx.x >> 5] = w;
    }
    __syncthreads();
    // thread q sums quantity q over the warps in order; every thread reads
    // the NV results
    __shared__ double r[NV];
    if (threadIdx.x < NV) {
        double u = 0.0;
        for (int w = 0; w < BT / 32; w++)
            u += s[threadIdx.x][w];
        r[threadIdx.x] = u;
    }
    __syncthreads();
    for (int q = 0; q < NV; q++)
        out[q] = r[q];
}

// mean and sigma (mat_mean_and_stddev, matrix_math.cpp:457-499):
// sum x, sum x^2 per block, then mean = sum / n and
// sigma = sqrt(sum x^2 / n - mean^2) in the last block.  Also clears the
// histogram bins for the binned median (when given).
template <typename T>
__global__ void __launch_bounds__(SF_THREADS, SF_STREAM_BLOCKS) k_sum_sq(const T* x, int64_t n, double* part,
    unsigned int* ticket, SfStats* st, unsigned long long* bins)
{
    double v[2] = { 0.0, 0.0 };
    for_each_elem(x, n, [&](double a) {
        v[0] += a;
        v[1] += a * a;
    });
    block_sums<2>(v, part + 2 * blockIdx.x);
    if (!last_block(ticket))
        return;
    double s[2];
    reduce_parts<2>(part, gridDim.x, s);
    if (bins)
        for (int k = threadIdx.x; k < BINS_N + 2; k += SF_THREADS)
            bins[k] = 0;
    if (threadIdx.x == 0) {
        const double dn = double(n);
        const double mean = __ddiv_rn(s[0], dn);
        st->mean = mean;
        st->sigma = __dsqrt_rn(__dsub_rn(__ddiv_rn(s[1], dn), __dmul_rn(mean, mean)));
    }
}

// The binned median from the merged bins (every thread of a block of BT
// threads calls it; the result is valid in every thread): the cumulative
// counts, consecutive bins per thread, locate the bin holding rank
// k = ceil(n / 2); for even n the walk continues over the bins whose
// cumulative count equals k, as the reference's loop does.  False when no
// bin reaches the rank.
template <int BT = SF_THREADS>
__device__ __forceinline__ bool hist_median(const unsigned long long* bins, int64_t n, double scale, double leftend,
    double* median)
{
    constexpr int BPT = (BINS_N + 1 + BT - 1) / BT; // bins per thread
    __shared__ unsigned long long cum[BPT * BT];
    __shared__ int hit;
    __shared__ double res;
    unsigned long long b4[BPT], loc = 0;
    for (int q = 0; q < BPT; q++) {
        const int i = BPT * threadIdx.x + q;
        b4[q] = i <= BINS_N ? __ldcg(bins + i) : 0ull;
        loc += b4[q];
    }
    if (threadIdx.x == 0)
        hit = -1;
    unsigned long long tot = 0;
    unsigned long long c = __ldcg(bins + BINS_N + 1) + block_excl_scan<BT>(loc, &tot);
    const unsigned long long k = (n & 1) ? (unsigned long long)(n + 1) / 2 : (unsigned long long)n / 2;
    for (int q = 0; q < BPT; q++) {
        const unsigned long long prev = c;
        c += b4[q];
        cum[BPT * threadIdx.x + q] = c;
        const int i = BPT * threadIdx.x + q;
        if (i <= BINS_N && c >= k && prev < k)
            hit = i; // exactly one bin crosses the rank
        if (i == 0 && prev >= k)
            hit = 0; // the count below the range already reaches it
    }
    __syncthreads();
    const int i = hit;
    if (threadIdx.x == 0 && i >= 0) {
        if (n & 1) {
            res = __dadd_rn(__ddiv_rn(double(i) + 0.5, scale), leftend);
        } else {
            unsigned long long count = cum[i];
            int j = i;
            while (count == k) {
                j++;
                count += __ldcg(bins + j);
                if (j == BINS_N)
                    break;
            }
            res = __dadd_rn(__ddiv_rn(double(i + j + 1), __dmul_rn(2.0, scale)), leftend);
        }
    }
    __syncthreads();
    *median = res;
    const bool ok = i >= 0;
    __syncthreads();
    return ok;
}

// mat_median_binapprox (matrix_math.cpp:334-455): N+1 bins over
// [mean - sigma, mean + sigma] plus the count below, bin = int((x - leftend)
// * scale), scale = N / (2 sigma); the last block walks the cumulative
// counts to the median's bin.  sigma * 2 < 1e-4, or no bin reaching the
// median's rank, set need_exact (the exact median is then taken instead).
template <typename T>
__global__ void __launch_bounds__(SF_THREADS, SF_STREAM_BLOCKS) k_hist(const T* x, int64_t n, SfStats* st,
    unsigned long long* bins /* BINS_N + 2: [0..N] bins, [N+1] bottom */, unsigned int* ticket)
{
    const double mean = st->mean, sigma = st->sigma;
    if (__dmul_rn(sigma, 2.0) < 0.0001) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            st->need_exact = 1;
        return;
    }
    const double scale = __ddiv_rn(double(BINS_N), __dmul_rn(2.0, sigma));
    const double leftend = __dsub_rn(mean, sigma);
    __shared__ unsigned int h[BINS_N + 2];
    for (int k = threadIdx.x; k < BINS_N + 2; k += blockDim.x)
        h[k] = 0;
    __syncthreads();
    for_each_elem(x, n, [&](double a) {
        const int b = int_trunc_x86(__dmul_rn(__dsub_rn(a, leftend), scale));
        if (b < 0)
            atomicAdd(&h[BINS_N + 1], 1u);
        else if (b <= BINS_N)
            atomicAdd(&h[b], 1u);
    });
    __syncthreads();
    for (int k = threadIdx.x; k < BINS_N + 2; k += blockDim.x)
        if (h[k])
            atomicAdd(&bins[k], (unsigned long long)h[k]);
    if (!last_block(ticket))
        return;
    double median;
    const bool ok = hist_median(bins, n, scale, leftend, &median);
    if (threadIdx.x == 0) {
        if (ok)
            st->median = median;
        else
            st->need_exact = 1;
    }
}

// Median from the exact (host-driven) selection.
__global__ void k_sf_set_median(SfStats* st, double median)
{
    st->median = median;
}

// -------------------------------------------------- exact selection (nth_element)

// Radix select, 16-bit digits over order keys.  pass: digit index 3..0
// (most significant first); prefix/mask select the candidates.
template <typename T>
__global__ void __launch_bounds__(SF_THREADS) k_radix_hist(const T* x, int64_t n, unsigned long long prefix,
    unsigned long long mask, int shift, unsigned int* hist /* 65536 */)
{
    for_each_elem(x, n, [&](double a) {
        const unsigned long long k = okey(a);
        if ((k & mask) == prefix)
            atomicAdd(&hist[(k >> shift) & 0xffffull], 1u);
    });
}

// Single block: find the digit bucket containing rank `state[0]` (0-based
// among candidates); update prefix/mask/rank in `state`
// (state: [0] rank, [1] prefix, [2] mask).
__global__ void k_radix_pick(const unsigned int* hist, int shift, unsigned long long* state)
{
    __shared__ unsigned long long s[1024];
    const unsigned long long rank = state[0]; // read before any thread updates it
    // each thread owns 64 consecutive digits
    unsigned long long loc = 0;
    const int d0 = threadIdx.x * 64;
    for (int k = 0; k < 64; k++)
        loc += hist[d0 + k];
    s[threadIdx.x] = loc;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        unsigned long long t = threadIdx.x >= o ? s[threadIdx.x - o] : 0ull;
        __syncthreads();
        s[threadIdx.x] += t;
        __syncthreads();
    }
    const unsigned long long incl = s[threadIdx.x], excl = incl - loc;
    if (rank >= excl && rank < incl) {
        unsigned long long c = excl;
        for (int k = 0; k < 64; k++) {
            const unsigned long long h = hist[d0 + k];
            if (rank < c + h) {
                state[0] = rank - c;
                state[1] |= (unsigned long long)(d0 + k) << shift;
                state[2] |= 0xffffull << shift;
                break;
            }
            c += h;
        }
    }
}

// -------------------------------------------------- sigma clip (estimate_rms)

// estimate_rms (sourcefind.cpp:54-134) with the iteration state on the
// device.  A clipping pass sums v, v^2 and the count of samples with
// |x - median| > upper and not > prev_upper; its last block sums the
// partials in a fixed order and updates the state exactly as the
// reference's loop (sourcefind.cpp:82-134), with explicitly rounded
// operations; once nothing is removed the remaining passes return at once.
struct ClipState {
    double s, d1, d2, valid, prev_upper, upper;
    int done;
};

// Starting state from the mean, sigma and median (m = mean - median).
__device__ __forceinline__ ClipState clip_start(double mean, double sigma, double median, double n, double num_sigma)
{
    const double m = __dsub_rn(mean, median);
    ClipState c;
    c.s = sigma;
    c.d1 = __dmul_rn(m, n);
    c.d2 = __dmul_rn(__dadd_rn(__dmul_rn(sigma, sigma), __dmul_rn(m, m)), n);
    c.valid = n;
    c.prev_upper = 1.7976931348623157e308;
    c.upper = __dmul_rn(num_sigma, sigma);
    c.done = 0;
    return c;
}

// One pass's update from the sums of the removed samples (sm: v, v^2,
// count), sourcefind.cpp:82-134.
__device__ __forceinline__ void clip_update(ClipState& c, const double* sm, double num_sigma)
{
    const unsigned long long rem = (unsigned long long)(sm[2] + 0.5);
    if (rem == 0) {
        c.done = 1;
        return;
    }
    c.valid = __dsub_rn(c.valid, double(rem));
    c.d1 = __dsub_rn(c.d1, sm[0]);
    c.d2 = __dsub_rn(c.d2, sm[1]);
    const double a = __ddiv_rn(c.d2, c.valid), b = __ddiv_rn(c.d1, c.valid);
    c.s = __dsqrt_rn(__dsub_rn(a, __dmul_rn(b, b)));
    c.prev_upper = c.upper;
    c.upper = __dmul_rn(num_sigma, c.s);
}

__global__ void k_clip_init(ClipState* cs, const SfStats* st, double n, double num_sigma)
{
    *cs = clip_start(st->mean, st->sigma, st->median, n, num_sigma);
}

template <typename T>
__global__ void __launch_bounds__(SF_THREADS, SF_STREAM_BLOCKS) k_clip_pass(const T* x, int64_t n, const SfStats* st,
    ClipState* cs, double* part, unsigned int* ticket, double num_sigma)
{
    if (cs->done)
        return;
    const double median = st->median;
    const double upper = cs->upper, prev_upper = cs->prev_upper;
    // Single-precision screen: samples with |x - median| certainly not above
    // upper skip the double-precision tests.  With xf = float(x), mf =
    // float(median), |x - median| <= |xf - mf| (1 + 2^-23) + |xf| 2^-23 +
    // |median| 2^-24, so |xf - mf| + |xf| 2^-21 < skip, skip <= upper
    // (1 - 2^-12) - |median| 2^-12, implies |x - median| < upper.  NaN and
    // infinite samples fail the screen and take the exact tests.
    const float mf = float(median);
    const float skip = __double2float_rd(upper * (1.0 - 0x1p-12) - fabs(median) * 0x1p-12);
    auto screened = [&](T xr) {
        const float xf = float(xr);
        return fabsf(xf - mf) + fabsf(xf) * 0x1p-21f < skip;
    };
    double v[3] = { 0.0, 0.0, 0.0 };
    auto band_exact = [&](double xv) {
        const double d = xv - median;
        const double a = fabs(d);
        if (a > upper && !(a > prev_upper)) {
            v[0] += d;
            v[1] += d * d;
            v[2] += 1.0;
        }
    };
    auto band = [&](T xr) {
        if (!screened(xr))
            band_exact(double(xr));
    };
    for_each_elem(x, n, band);
    block_sums<3>(v, part + 3 * blockIdx.x);
    if (!last_block(ticket))
        return;
    double sm[3];
    reduce_parts<3>(part, gridDim.x, sm);
    if (threadIdx.x != 0)
        return;
    ClipState c = *cs;
    clip_update(c, sm, num_sigma);
    *cs = c;
}

__device__ __host__ inline uint32_t fkey32(float v);

// rms (the clipped sigma, or the caller's estimate when cs is null) and the
// thresholds bg +- n_sigma * rms with bg = the median (sourcefind.cpp:298-301),
// with the detection thresholds' keys for the label analysis: order keys,
// and for single-precision images the largest float <= the positive
// threshold and the smallest float >= the negative one.
__device__ __forceinline__ void sf_set_thresholds(SfStats* st, double rms, double ana, double det)
{
    const double bg = st->median;
    st->rms = rms;
    st->thr[0] = __dadd_rn(bg, __dmul_rn(ana, rms));
    st->thr[1] = __dsub_rn(bg, __dmul_rn(ana, rms));
    const double dp = __dadd_rn(bg, __dmul_rn(det, rms)), dn = __dsub_rn(bg, __dmul_rn(det, rms));
    st->thr[2] = dp;
    st->thr[3] = dn;
    st->kpos = okey(dp);
    st->kneg = okey(dn);
    float tf = __double2float_rn(dp);
    if (double(tf) > dp)
        tf = nextafterf(tf, -INFINITY);
    float tc = __double2float_rn(dn);
    if (double(tc) < dn)
        tc = nextafterf(tc, INFINITY);
    st->fpos = fkey32(tf);
    st->fneg = fkey32(tc);
}

__global__ void k_sf_thresholds(SfStats* st, const ClipState* cs, double rms_fixed, double ana, double det)
{
    sf_set_thresholds(st, cs ? cs->s : rms_fixed, ana, det);
}

// -------------------------------------------------- fused statistics (one cooperative launch)

// Polls of a grid barrier before it gives up (each poll sleeps ~32 ns; a
// legitimate wait is one pass over the image, tens of microseconds).
constexpr uint32_t kGridWaitLimit = 1u << 20;

// Grid-wide barrier of a cooperative launch (every block resident): the
// k-th arrival of each block adds one to *count and waits until it reaches
// k * gridDim.x.  Writes before the barrier are visible after it (fence,
// then acquire loads; readers use L2 loads).  A wait that runs out records
// the failure in *err and returns false in the whole block; the caller's
// kernel then ends, and so does every other block's at its next wait.
__device__ __forceinline__ bool grid_barrier(unsigned int* count, unsigned int target, unsigned int* err)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(count, 1u);
        int good = 0;
        for (uint32_t it = 0; it < kGridWaitLimit; it++) {
            unsigned int v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if (v >= target) {
                good = 1;
                break;
            }
            __nanosleep(32);
        }
        if (!good)
            atomicExch(err, 1u);
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Lower edge of a full clip pass's band, as a fraction of its threshold:
// the samples with kClipBand * upper < |x - median| <= upper are kept for
// the passes that follow.
constexpr double kClipBand = 0.8;

// Capacity of a thread's band list in k_sf_stats for n samples over G
// threads (a quarter of the thread's samples, plus slack).
__host__ __device__ inline int sf_band_cap(int64_t n, int64_t G)
{
    const int64_t per_thread = 4 * ((n / 4 + G - 1) / G) + 1;
    return int(per_thread / 4 + 4);
}

// Threads of a k_sf_stats block; one block per SM.
constexpr int SF_STATS_THREADS = 1024;

// Histogram slot of a single-precision sample for the binned median without
// double-precision arithmetic where that is safe; the slot is that of
// int_trunc_x86((double(x) - leftend) * scale) in double precision (bins 0..N,
// N + 1 = below the range).  With lf = float(leftend), sf = float(scale), tf =
// (x - lf) * sf in single precision differs from the exact t = (x - leftend)
// * scale by at most 2^-22 (|tf| + |leftend| scale) (three roundings of 2^-24
// each on the terms, one of 2^-24 |leftend| from lf); e = 2^-20 |tf| + els,
// els >= 2^-20 |leftend| scale, covers that and the roundings of tf -+ e.
// When [tf - e, tf + e] holds no bin edge the slot follows from it: below
// (t < -1), bin 0 (-1 < t < 1: truncation), the bin of floor (through the
// 1.5 * 2^23 rounding constant), or none (N + 1 <= t < 2^30; beyond 2^31 the
// truncation's integer-indefinite value counts as below, so large t are not
// decided here).  Returns the slot, -2 for none, -3 when undecided (an edge
// in the interval, NaN or infinite samples): the caller then takes the
// double-precision path.  Straight-line code: the rare -3 is the only branch
// a warp may split on.
__device__ __forceinline__ int fast_bin(float x, float lf, float sf, float els)
{
    const float tf = __fmul_rn(__fsub_rn(x, lf), sf);
    const float e = __fmaf_rn(fabsf(tf), 0x1p-20f, els);
    const float lo = __fsub_rn(tf, e), hi = __fadd_rn(tf, e);
    constexpr float M = 12582912.0f; // 1.5 * 2^23: adding it rounds to an integer
    const float hm = __fadd_rn(hi, M);
    const float rf = __fsub_rn(hm, M);
    const bool up = rf > hi;
    const float fl = up ? __fsub_rn(rf, 1.0f) : rf;
    const int fi = __float_as_int(hm) - 0x4B400000 - (up ? 1 : 0);
    const bool below = hi < -1.0f;
    const bool none = lo >= float(BINS_N + 1) && hi < 0x1p30f;
    const bool in = lo > -1.0f && hi < float(BINS_N + 1) && (hi < 1.0f || fmaxf(lo, 0.0f) >= fl);
    return below ? BINS_N + 1 : in ? max(fi, 0) : none ? -2 : -3;
}

// Statistics and thresholds of the source finder in one cooperative launch
// of one SF_STATS_THREADS block per SM (sourcefind.cpp:280-301): sum x and
// x^2 (mean, sigma; do_sum), the binned median (do_hist; otherwise the
// median already in st), clip_iters sigma-clip passes (estimate_rms; none
// when the caller gives the rms), the thresholds.  Grid barriers separate
// the steps, and after each every block reduces all blocks' partials in the
// same fixed order, so every block holds the same statistics and takes the
// same branches; the arithmetic of each step is that of the pass kernels
// above (the histogram of single-precision images through fast_bin, which
// gives the same bins).  A full clip pass keeps, per thread, its samples
// with kClipBand * upper < |x - median| <= upper in a private list
// (cand[k * G + thread], k < cap), and a later pass whose threshold is still
// above the band's lower edge visits only those lists: it removes the
// samples with upper' < |x - median| <= prev_upper, and prev_upper <= the
// full pass's upper (thresholds fall while passes remove samples), so all
// of them are listed.  A list that would overflow is counted in a fourth
// partial and the next pass reads the image again.  Failures: the binned
// median not applying sets need_exact (and thresholds that label nothing); a
// barrier that gives up sets stats_err.
template <typename T>
__global__ void __launch_bounds__(SF_STATS_THREADS, 1) k_sf_stats(const T* x, int64_t n, SfStats* st,
    ClipState* cs, double* part /* 2 * 4 * gridDim.x */, unsigned long long* bins /* BINS_N + 2 */, T* cand, int cap,
    unsigned int* bar, int do_sum, int do_hist, int clip_iters, double rms_fixed, double ana, double det)
{
    constexpr int BT = SF_STATS_THREADS;
    const int nb = gridDim.x;
    const int64_t G = int64_t(nb) * BT, gt = int64_t(blockIdx.x) * BT + threadIdx.x;
    const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
    const double dn = double(n);
    unsigned int arrivals = 0;
    auto sync = [&]() {
        arrivals++;
        return grid_barrier(bar, arrivals * unsigned(nb), &st->stats_err);
    };
    int step = 0;
    auto next_part = [&]() { return part + 4 * int64_t(nb) * (step++ & 1); };
    auto label_nothing = [&]() {
        if (lead) {
            st->need_exact = 1;
            sf_set_thresholds(st, INFINITY, ana, det);
        }
    };
    double mean = st->mean, sigma = st->sigma, median = st->median;
    if (do_sum) {
        double v[2] = { 0.0, 0.0 };
        for_each_elem(x, n, [&](double a) {
            v[0] += a;
            v[1] += a * a;
        });
        double* pp = next_part();
        block_sums<2, BT>(v, pp + 2 * blockIdx.x);
        if (do_hist && blockIdx.x == 0)
            for (int k = threadIdx.x; k < BINS_N + 2; k += BT)
                bins[k] = 0;
        if (!sync())
            return;
        double s2[2];
        reduce_parts<2, BT>(pp, nb, s2);
        mean = __ddiv_rn(s2[0], dn);
        sigma = __dsqrt_rn(__dsub_rn(__ddiv_rn(s2[1], dn), __dmul_rn(mean, mean)));
        if (lead) {
            st->mean = mean;
            st->sigma = sigma;
        }
    }
    if (do_hist) {
        if (__dmul_rn(sigma, 2.0) < 0.0001) {
            label_nothing();
            return;
        }
        const double scale = __ddiv_rn(double(BINS_N), __dmul_rn(2.0, sigma));
        const double leftend = __dsub_rn(mean, sigma);
        // four copies of the bins (warp w adds to copy w % 4), summed at the end
        constexpr int HB = BINS_N + 2;
        __shared__ unsigned int h[4 * HB];
        for (int k = threadIdx.x; k < 4 * HB; k += BT)
            h[k] = 0;
        __syncthreads();
        unsigned int* hw = h + HB * ((threadIdx.x >> 5) & 3);
        auto exact_bin = [&](double a) {
            const int b = int_trunc_x86(__dmul_rn(__dsub_rn(a, leftend), scale));
            if (b <= BINS_N)
                atomicAdd(&hw[b < 0 ? BINS_N + 1 : b], 1u);
        };
        if constexpr (sizeof(T) == 4) {
            const float lf = __double2float_rn(leftend), sf = __double2float_rn(scale);
            const float els = __double2float_ru(fabs(leftend) * scale * 0x1p-20);
            for_each_elem(x, n, [&](T xr) {
                const int b = fast_bin(xr, lf, sf, els);
                if (b >= 0)
                    atomicAdd(&hw[b], 1u);
                else if (b == -3)
                    exact_bin(double(xr));
            });
        } else {
            for_each_elem(x, n, [&](double a) { exact_bin(a); });
        }
        __syncthreads();
        for (int k = threadIdx.x; k < HB; k += BT) {
            const unsigned int c = h[k] + h[HB + k] + h[2 * HB + k] + h[3 * HB + k];
            if (c)
                atomicAdd(&bins[k], (unsigned long long)c);
        }
        if (!sync())
            return;
        if (!hist_median<BT>(bins, n, scale, leftend, &median)) {
            label_nothing();
            return;
        }
        if (lead)
            st->median = median;
    }
    double rms = rms_fixed;
    if (clip_iters > 0) {
        ClipState c = clip_start(mean, sigma, median, dn, 3.0);
        const float mf = float(median);
        int cnt = 0; // this thread's listed samples
        double list_lo = INFINITY; // lower edge of the lists' band (none yet)
        for (int it = 0; it < clip_iters && !c.done; it++) {
            const double upper = c.upper, prev_upper = c.prev_upper;
            double v[4] = { 0.0, 0.0, 0.0, 0.0 };
            auto band_exact = [&](double xv) {
                const double d = xv - median;
                const double a = fabs(d);
                if (a > upper && !(a > prev_upper)) {
                    v[0] += d;
                    v[1] += d * d;
                    v[2] += 1.0;
                }
            };
            if (upper >= list_lo) {
                for (int k = 0; k < cnt; k++)
                    band_exact(double(cand[int64_t(k) * G + gt]));
            } else {
                // full pass; the single-precision screen of k_clip_pass at
                // the band's lower edge
                const double lo = kClipBand * upper;
                const float skip = __double2float_rd(lo * (1.0 - 0x1p-12) - fabs(median) * 0x1p-12);
                int m = 0;
                auto visit = [&](T xr) {
                    const double xv = double(xr);
                    band_exact(xv);
                    const double a = fabs(xv - median);
                    if (a > lo && !(a > upper)) {
                        if (m < cap)
                            cand[int64_t(m) * G + gt] = xr;
                        m++;
                    }
                };
                auto fails = [&](T xr) {
                    const float xf = float(xr);
                    return !(fabsf(xf - mf) + fabsf(xf) * 0x1p-21f < skip);
                };
                // the screen over a step's samples first, then the samples
                // that fail it (re-read), so that a warp splits once a step
                // rather than once a sample
                constexpr int UNR = sizeof(T) == 4 ? 4 : 2;
                const int64_t n4 = n / 4;
                int64_t g = gt;
                for (; g + (UNR - 1) * G < n4; g += UNR * G) {
                    T a[UNR][4];
#pragma unroll
                    for (int u = 0; u < UNR; u++)
                        load4(x, g + u * G, a[u]);
                    unsigned int fm = 0;
#pragma unroll
                    for (int u = 0; u < UNR; u++)
#pragma unroll
                        for (int k = 0; k < 4; k++)
                            fm |= (fails(a[u][k]) ? 1u : 0u) << (4 * u + k);
                    while (fm) {
                        const int slot = __ffs(fm) - 1;
                        fm &= fm - 1;
                        visit(x[4 * (g + (slot >> 2) * G) + (slot & 3)]);
                    }
                }
                for (; g < n4; g += G) {
                    T a[4];
                    load4(x, g, a);
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (fails(a[k]))
                            visit(a[k]);
                }
                for (int64_t i = n4 * 4 + gt; i < n; i += G)
                    if (fails(x[i]))
                        visit(x[i]);
                cnt = m < cap ? m : cap;
                v[3] = m > cap ? 1.0 : 0.0;
                list_lo = lo;
            }
            double* pp = next_part();
            block_sums<4, BT>(v, pp + 4 * blockIdx.x);
            if (!sync())
                return;
            double sm[4];
            reduce_parts<4, BT>(pp, nb, sm);
            if (sm[3] > 0.0)
                list_lo = INFINITY; // a list overflowed: the next pass reads the image
            clip_update(c, sm, 3.0);
        }
        rms = c.s;
        if (lead)
            *cs = c;
    }
    if (lead)
        sf_set_thresholds(st, rms, ana, det);
}

// -------------------------------------------------- connected components

// Scan key of memory pixel (mr, mc): the reference scans display columns
// c_i = (mc + cols/2) mod cols in order, rows in memory order (ccl.h:162-183).
struct CclGeom {
    int rows, cols, rshift, cshift;
    // images hold fewer than 2^32 pixels (checked by the callers), so the
    // index arithmetic is 32-bit
    __device__ __forceinline__ int64_t mem_of_key(int64_t s) const
    {
        const uint32_t su = uint32_t(s), ur = uint32_t(rows);
        const int ci = int(su / ur), r = int(su - uint32_t(ci) * ur);
        const int mc = ci >= cshift ? ci - cshift : ci + cshift;
        return int64_t(mc) * rows + r;
    }
};

// The labelling passes after the first work on chunks of CCL_CHUNK scan keys,
// one block of SF_THREADS threads per chunk, each thread reading the classes
// of CCL_KPT consecutive keys with one 16-byte load.  The class array is
// padded with background up to a whole number of chunks.
constexpr int CCL_KPT = 16;
constexpr int CCL_CHUNK = SF_THREADS * CCL_KPT;

__device__ __forceinline__ uint32_t cls_at(const uint32_t (&w)[4], int k)
{
    return (w[k >> 2] >> (8 * (k & 3))) & 0xffu;
}

__device__ __forceinline__ void load_cls16(const uint8_t* cls, uint32_t (&w)[4])
{
    const uint4 v = reinterpret_cast<const uint4*>(cls)[int64_t(blockIdx.x) * SF_THREADS + threadIdx.x];
    w[0] = v.x;
    w[1] = v.y;
    w[2] = v.z;
    w[3] = v.w;
}

// The chunk's foreground keys in scan order, compacted into q as
// (offset in the chunk) | class << 12; returns their number.
__device__ __forceinline__ int chunk_queue(const uint32_t (&w)[4], uint16_t* q)
{
    uint32_t mask = 0;
#pragma unroll
    for (int k = 0; k < CCL_KPT; k++)
        if (cls_at(w, k))
            mask |= 1u << k;
    unsigned long long tot = 0;
    int p = int(block_excl_scan(__popc(mask), &tot));
    while (mask) {
        const int k = __ffs(mask) - 1;
        mask &= mask - 1;
        q[p++] = uint16_t((threadIdx.x * CCL_KPT + k) | (cls_at(w, k) << 12));
    }
    __syncthreads();
    return int(tot);
}

// Classes (0 background, 1 above the positive analysis threshold, 2 below
// the negative one) and parents of foreground keys, one key per thread; the
// general form, for any even image size.  The thresholds are thr[0], thr[1]
// when thr is given (computed on the device), else tp, tn.
template <typename T>
__global__ void k_ccl_init(const T* img, CclGeom g, const double* thr, double tp, double tn, int findneg, uint8_t* cls,
    uint32_t* P)
{
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t n = int64_t(g.rows) * g.cols;
    if (s >= n)
        return;
    if (thr) {
        tp = thr[0];
        tn = thr[1];
    }
    const double v = ld(img, g.mem_of_key(s));
    uint8_t c = 0;
    if (v > tp)
        c = 1;
    else if (findneg && v < tn)
        c = 2;
    cls[s] = c;
    if (c)
        P[s] = uint32_t(s);
}

// The same for rows % 4 == 0 and a 16-byte aligned image: CCL_KPT keys per
// step in groups of four keys of one column (one 16-byte load each, or two
// for doubles, all issued before the classes are formed), classes stored
// as one 16-byte word, parents of groups holding foreground as one 16-byte
// store.  Groups from ngroups on are the background padding of the class
// array (nunits = its length in CCL_KPT keys).
template <typename T>
__global__ void __launch_bounds__(SF_THREADS) k_ccl_init16(const T* img, CclGeom g, const double* thr, double tp,
    double tn, int findneg, int64_t ngroups, int64_t nunits, uint4* cls16, uint4* P4)
{
    if (thr) {
        tp = thr[0];
        tn = thr[1];
    }
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < nunits; u += stride) {
        T v[16];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t q = 4 * u + j;
            if (q < ngroups) {
                T a[4];
                load4(img + g.mem_of_key(4 * q), 0, a);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    v[4 * j + k] = a[k];
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++)
                    v[4 * j + k] = T(0);
            }
        }
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            uint32_t packed = 0;
            if (4 * u + j < ngroups) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const double x = double(v[4 * j + k]);
                    uint32_t c = 0;
                    if (x > tp)
                        c = 1;
                    else if (findneg && x < tn)
                        c = 2;
                    packed |= c << (8 * k);
                }
            }
            if (packed) {
                const uint32_t s = uint32_t(16 * u + 4 * j);
                P4[4 * u + j] = make_uint4(s, s + 1, s + 2, s + 3);
            }
            w[j] = packed;
        }
        cls16[u] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

__device__ __forceinline__ uint32_t uf_find(const uint32_t* P, uint32_t x, unsigned* err)
{
    for (uint32_t it = 0; it < UF_MAX_STEPS; it++) {
        const uint32_t y = P[x];
        if (y == x)
            return x;
        x = y;
    }
    atomicOr(err, 2u);
    return x;
}

// Lock-free union by minimum root (links the larger root under the smaller),
// so every component's root is its smallest scan key.
__device__ __forceinline__ void uf_union(uint32_t* P, uint32_t a, uint32_t b, unsigned* err)
{
    for (uint32_t it = 0; it < UF_MAX_STEPS; it++) {
        a = uf_find(P, a, err);
        b = uf_find(P, b, err);
        if (a == b)
            return;
        if (a < b) {
            const uint32_t old = atomicMin(&P[b], a);
            if (old == b)
                return;
            b = old;
        } else {
            const uint32_t old = atomicMin(&P[a], b);
            if (old == a)
                return;
            a = old;
        }
    }
    atomicOr(err, 4u);
}

// Links of the reference's labeling graph, non-FFTSHIFT build
// (ccl.h:162-342 scan + row border merge, :355-448 column border merge;
// 4-connectivity :545-745).  With s = (c_i, r):
//   left       (c_i-1, r)                      c_i >= 1
//   top        (c_i, r-1)                      r not in {0, rows/2}
//   row wrap   (c_i, rows-1)                   r == 0
//   8-conn only:
//   top-left   (c_i-1, r-1)                    c_i >= 1, r not in {0, rows/2}
//   bottom-left(c_i-1, r+1)                    c_i >= 1, r not in {rows/2-1, rows-1}
//   wrap t-left(c_i-1, rows-1)                 c_i >= 1, r == 0
//   slice link (c_i-1, 0)                      r == rows-1, c_i a slice start
// One thread per foreground key of the chunk (compacted first, so the
// unions of a dense island run in parallel).
__global__ void __launch_bounds__(SF_THREADS) k_ccl_union(const uint8_t* cls, CclGeom g, int conn4, int slice_cols,
    uint32_t* P, unsigned* err)
{
    __shared__ uint16_t q[CCL_CHUNK];
    uint32_t w[4];
    load_cls16(cls, w);
    const int nq = chunk_queue(w, q);
    const int64_t base = int64_t(blockIdx.x) * CCL_CHUNK;
    const int rows = g.rows;
    for (int i = threadIdx.x; i < nq; i += SF_THREADS) {
        const int64_t s = base + (q[i] & 0xfff);
        const uint32_t my = q[i] >> 12;
        const int ci = int(uint32_t(s) / uint32_t(rows)), r = int(uint32_t(s) - uint32_t(ci) * uint32_t(rows));
        auto link = [&](int64_t t) {
            if (cls[t] == my)
                uf_union(P, uint32_t(s), uint32_t(t), err);
        };
        if (ci >= 1)
            link(s - rows);
        if (r != 0 && r != g.rshift)
            link(s - 1);
        if (r == 0)
            link(s + rows - 1);
        if (!conn4 && ci >= 1) {
            if (r != 0 && r != g.rshift)
                link(s - rows - 1);
            if (r != g.rshift - 1 && r != rows - 1)
                link(s - rows + 1);
            if (r == 0)
                link(s - 1);
            if (r == rows - 1 && (ci % slice_cols) == 0)
                link(s - 2 * int64_t(rows) + 1);
        }
    }
}

// Path compression of every foreground key to its root, and per chunk the
// number of positive roots, negative roots and foreground keys (rows 0, 1,
// 2 of cnt, row stride `stride`).
__global__ void __launch_bounds__(SF_THREADS) k_ccl_flatten(const uint8_t* cls, uint32_t* P, uint32_t* cnt, int stride,
    unsigned* err)
{
    __shared__ uint16_t q[CCL_CHUNK];
    uint32_t w[4];
    load_cls16(cls, w);
    const int nq = chunk_queue(w, q);
    const uint32_t base = uint32_t(blockIdx.x) * CCL_CHUNK;
    uint32_t rp = 0, rn = 0;
    for (int i = threadIdx.x; i < nq; i += SF_THREADS) {
        const uint32_t s = base + (q[i] & 0xfff);
        const uint32_t r = uf_find(P, s, err);
        if (r == s) {
            if ((q[i] >> 12) == 1)
                rp++;
            else
                rn++;
        } else {
            P[s] = r;
        }
    }
    unsigned long long tot = 0;
    block_excl_scan(rp | (unsigned long long)rn << 16, &tot);
    if (threadIdx.x == 0) {
        cnt[blockIdx.x] = uint32_t(tot & 0xffff);
        cnt[stride + blockIdx.x] = uint32_t((tot >> 16) & 0xffff);
        cnt[2 * stride + blockIdx.x] = uint32_t(nq);
    }
}

// Final label number of each root: 1 + its rank among roots of the same sign
// in scan order (ccl.h:452-480 numbers roots in increasing provisional-label
// order, which is scan order of each component's first pixel); off holds the
// exclusive scans of k_ccl_flatten's counts.  With fgl, also the list of all
// foreground keys in scan order.
__global__ void __launch_bounds__(SF_THREADS) k_ccl_rank(const uint8_t* cls, const uint32_t* P, const uint32_t* off,
    int stride, uint32_t* R, uint32_t* fgl)
{
    uint32_t w[4];
    load_cls16(cls, w);
    const uint32_t s0 = uint32_t(blockIdx.x) * CCL_CHUNK + threadIdx.x * CCL_KPT;
    uint32_t fgmask = 0, rootmask = 0, np = 0, nn = 0;
#pragma unroll
    for (int k = 0; k < CCL_KPT; k++) {
        const uint32_t c = cls_at(w, k);
        if (c) {
            fgmask |= 1u << k;
            if (P[s0 + k] == s0 + k) {
                rootmask |= 1u << k;
                if (c == 1)
                    np++;
                else
                    nn++;
            }
        }
    }
    unsigned long long tot = 0;
    const unsigned long long ex
        = block_excl_scan(np | (unsigned long long)nn << 16 | (unsigned long long)__popc(fgmask) << 32, &tot);
    uint32_t rp = off[blockIdx.x] + uint32_t(ex & 0xffff);
    uint32_t rn = off[stride + blockIdx.x] + uint32_t((ex >> 16) & 0xffff);
    uint32_t fp = off[2 * stride + blockIdx.x] + uint32_t(ex >> 32);
    while (fgmask) {
        const int k = __ffs(fgmask) - 1;
        fgmask &= fgmask - 1;
        const uint32_t s = s0 + k;
        if (rootmask & (1u << k))
            R[s] = cls_at(w, k) == 1 ? ++rp : ++rn;
        if (fgl)
            fgl[fp++] = s;
    }
}

// Label map in memory order: +rank (positive) / -rank (negative), 0 = background.
__global__ void k_ccl_label(const uint8_t* cls, const uint32_t* P, const uint32_t* R, CclGeom g, int32_t* L)
{
    const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t n = int64_t(g.rows) * g.cols;
    if (s >= n)
        return;
    const int64_t m = g.mem_of_key(s);
    const uint8_t c = cls[s];
    L[m] = c == 0 ? 0 : (c == 1 ? int32_t(R[P[s]]) : -int32_t(R[P[s]]));
}

// The same CCL_KPT keys at a time in groups of four keys of one column
// (rows % 4 == 0, 16-byte aligned label map): one 16-byte class load and four
// 16-byte stores per step; the label lookups of a step are independent.
__global__ void __launch_bounds__(SF_THREADS) k_ccl_label16(const uint8_t* cls, const uint32_t* P, const uint32_t* R,
    CclGeom g, int64_t ngroups, int32_t* L)
{
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    const int64_t nunits = (ngroups + 3) / 4;
    for (int64_t u = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; u < nunits; u += stride) {
        const uint4 c16 = reinterpret_cast<const uint4*>(cls)[u];
        const uint32_t cw[4] = { c16.x, c16.y, c16.z, c16.w };
        int v[16];
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const uint32_t c = (cw[k >> 2] >> (8 * (k & 3))) & 0xffu;
            v[k] = 0;
            if (c) {
                const int r = int(R[P[16 * u + k]]);
                v[k] = c == 1 ? r : -r;
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t q = 4 * u + j;
            if (q < ngroups)
                reinterpret_cast<int4*>(L)[g.mem_of_key(4 * q) >> 2]
                    = make_int4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        }
    }
}

// -------------------------------------------------- label analysis
//
// The stage is enqueued before the host knows its sizes: FgSizes reads the
// label counts and the foreground-list length from the labeller's counters
// and caps them at the capacities the buffers were sized for (the host runs
// the stage again with larger buffers when a cap was hit).  The kernels loop
// over their entries with a fixed grid.
//
// Everything after the labelling works on the list of foreground keys in
// scan order (k_ccl_rank's fgl), not on the image: entry i has the label
// code (positives 0..np-1, negatives np..np+nn-1) and the memory index of
// its pixel.

struct FgSizes {
    const uint32_t* misc; // [0] positive labels, [1] negative labels, [2] foreground entries
    uint32_t label_cap, fg_cap;
    __device__ __forceinline__ int np() const { return int(misc[0]); }
    __device__ __forceinline__ uint32_t nl() const { return min(misc[0] + misc[1], label_cap); }
    __device__ __forceinline__ uint32_t nfg() const { return min(misc[2], fg_cap); }
    __device__ __forceinline__ bool capped() const { return misc[0] + misc[1] > label_cap || misc[2] > fg_cap; }
};

#define FG_LOOP(i, count)                                                                                            \
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, i##_n = (count); i < i##_n; i += gridDim.x * blockDim.x)

// Single-precision images keep the extremum and its first memory index as
// one 64-bit key per label (the value's order key above the index;
// positives keep the maximum with the lowest index through atomicMax on
// ~index, negatives the minimum with the lowest index through atomicMin).
// Starting keys hold the detection threshold rounded to the float grid
// (largest float <= threshold for positives, smallest float >= threshold for
// negatives), so only values strictly beyond the threshold replace them.
__device__ __host__ inline uint32_t fkey32(float v)
{
    uint32_t u;
    memcpy(&u, &v, 4);
    return (u >> 31) ? ~u : (u | 0x80000000u);
}
__device__ inline float fkey32_inv(uint32_t k)
{
    const uint32_t u = (k >> 31) ? (k & 0x7fffffffu) : ~k;
    return __uint_as_float(u);
}

// Per-label starting state: extremum keys at the detection threshold
// (sourcefind.cpp:342-378 starts from it and compares strictly; PACKED: the
// value-and-index keys), first indices unset (eidx, when given), empty
// segments.
template <bool PACKED>
__global__ void k_fg_init(FgSizes z, const SfStats* st, unsigned long long* ext, unsigned long long* eidx,
    uint32_t* seg_begin, uint32_t* seg_end, uint32_t* seg_split)
{
    const int np = z.np();
    const unsigned long long vpos = PACKED ? (unsigned long long)st->fpos << 32 | 0xffffffffull : st->kpos;
    const unsigned long long vneg = PACKED ? (unsigned long long)st->fneg << 32 : st->kneg;
    FG_LOOP(i, z.nl())
    {
        ext[i] = int(i) < np ? vpos : vneg;
        if (eidx)
            eidx[i] = ~0ull;
        seg_begin[i] = 0;
        seg_end[i] = 0;
        seg_split[i] = 0;
    }
}

// Label code and memory index of each foreground key, and the extremum of
// each label: PACKED (single precision) the 64-bit value-and-index keys
// above, else the order key of the value (its first index follows in
// k_fg_extrema_idx).
template <typename T, bool PACKED>
__global__ void k_fg_gather(FgSizes z, const T* img, const uint8_t* cls, const uint32_t* P, const uint32_t* R,
    CclGeom g, const uint32_t* fgl, uint32_t* fcode, uint32_t* fm, unsigned long long* ext)
{
    const uint32_t np = uint32_t(z.np());
    FG_LOOP(i, z.nfg())
    {
        const uint32_t s = fgl[i];
        const bool pos = cls[s] == 1;
        const uint32_t r = R[P[s]] - 1;
        const uint32_t code = pos ? r : np + r;
        const uint32_t m = uint32_t(g.mem_of_key(s));
        fcode[i] = code;
        fm[i] = m;
        if (code >= z.label_cap)
            continue; // over capacity: the host runs the stage again
        if constexpr (PACKED) {
            const unsigned long long k = (unsigned long long)fkey32(float(img[m])) << 32;
            if (pos)
                atomicMax(&ext[code], k | (0xffffffffu - m));
            else
                atomicMin(&ext[code], k | m);
        } else {
            const unsigned long long k = okey(ld(img, m));
            if (pos)
                atomicMax(&ext[code], k);
            else
                atomicMin(&ext[code], k);
        }
    }
}

// First memory index holding the extremum (the serial reference keeps the
// first occurrence in memory order).
template <typename T>
__global__ void k_fg_extrema_idx(FgSizes z, const SfStats* st, const T* img, const uint32_t* fcode, const uint32_t* fm,
    const unsigned long long* ext, unsigned long long* eidx)
{
    const int np = z.np();
    const unsigned long long kpos = st->kpos, kneg = st->kneg;
    FG_LOOP(i, z.nfg())
    {
        const uint32_t code = fcode[i], m = fm[i];
        if (code >= z.label_cap)
            continue;
        const unsigned long long k = okey(ld(img, m));
        const bool hit = int(code) < np ? k > kpos : k < kneg;
        if (hit && k == ext[code])
            atomicMin(&eidx[code], (unsigned long long)m);
    }
}

// Entries of labels whose extremum passes the detection threshold, as 64-bit
// keys (label code above the list position) appended at an atomic cursor;
// pixels of the other labels are zeroed in the label map L when given
// (generate_labelmap).  PACKED: ext holds the single-precision
// value-and-index keys, which pass when their value part left the starting
// threshold (thr_pos / thr_neg); else the order keys of the extrema,
// compared with the detection keys.
template <bool PACKED>
__global__ void k_fg_keys(FgSizes z, const SfStats* st, const uint32_t* fcode, const uint32_t* fm,
    const unsigned long long* ext, unsigned long long* keys, uint32_t* count, int32_t* L, uint32_t* seg_count)
{
    const int np = z.np();
    // over capacity the validity is not final (the host runs the stage
    // again): the label map is left untouched until then
    if (z.capped())
        L = nullptr;
    FG_LOOP(i, z.nfg())
    {
        const uint32_t code = fcode[i];
        if (code >= z.label_cap)
            continue;
        const bool pos = int(code) < np;
        bool valid;
        if constexpr (PACKED)
            valid = uint32_t(ext[code] >> 32) != (pos ? st->fpos : st->fneg);
        else
            valid = pos ? ext[code] > st->kpos : ext[code] < st->kneg;
        if (valid) {
            keys[atomicAdd(count, 1u)] = (unsigned long long)code << 32 | i;
            atomicAdd(&seg_count[code], 1u); // the label's valid entries (k_seg_alloc)
        } else if (L) {
            L[fm[i]] = 0;
        }
    }
}

// Deterministic moments (sourcefind.cpp:457-569).  Sorted by key, the valid
// entries form one segment per label in list (scan) order.  Scan order visits
// the memory columns from cols/2 first, so a segment is memory order rotated:
// its pixels in memory columns < cols/2 (memory index < split_m) start at
// seg_split.  Memory order is [split, end) then [begin, split) -- the order
// of the reference's single-range loop.  seg_mark records, for sorted entry
// t of cnt, its memory index and the segment bounds it opens or closes.
__device__ __forceinline__ void seg_mark(const unsigned long long* k, uint32_t t, uint32_t cnt, const uint32_t* fm,
    uint32_t split_m, uint32_t* vals, uint32_t* seg_begin, uint32_t* seg_end, uint32_t* seg_split)
{
    const unsigned long long key = k[t];
    const uint32_t code = uint32_t(key >> 32), m = fm[uint32_t(key)];
    vals[t] = m;
    const bool first = t == 0 || uint32_t(k[t - 1] >> 32) != code;
    const bool last = t == cnt - 1 || uint32_t(k[t + 1] >> 32) != code;
    if (first)
        seg_begin[code] = t;
    if (last)
        seg_end[code] = t + 1;
    const bool low = m < split_m;
    if (low && (first || fm[uint32_t(k[t - 1])] >= split_m))
        seg_split[code] = t;
    if (!low && last)
        seg_split[code] = t + 1;
}

// seg_mark over keys sorted by the multi-block sort (the fall-back for a
// label above SEG_BIG valid entries).
__global__ void k_seg_mark(const unsigned long long* keys, uint32_t cnt, const uint32_t* fm, uint32_t split_m,
    uint32_t* vals, uint32_t* seg_begin, uint32_t* seg_end, uint32_t* seg_split)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < cnt)
        seg_mark(keys, t, cnt, fm, split_m, vals, seg_begin, seg_end, seg_split);
}

// Segments without a global sort.  The segments of the valid labels need
// not lie in label order (k_label_sums reads each label's own range), only
// each segment's entries in list (scan) order.  k_seg_alloc turns the
// per-label counts (in seg_end, from k_fg_keys) into ranges taken from an
// atomic cursor; k_seg_scatter drops every valid entry into its label's
// range; k_seg_sort orders each range by list position -- one warp per
// label (shuffles up to 32 entries, the warp's shared memory up to
// SEG_WARP), larger ranges queued for k_seg_sort_big (one block, up to
// SEG_BIG), above that the flag for the host's multi-block sort -- and writes
// the memory indices and the split point (the layout seg_mark gives the
// multi-block sort's result).
constexpr int SEG_WARP = 256;
constexpr int SEG_BIG = 16384;

// (the labels with entries are also listed, for k_seg_sort: alloc[1] of them)
__global__ void k_seg_alloc(FgSizes z, uint32_t* seg_begin, uint32_t* seg_end, uint32_t* cursor, uint32_t* alloc,
    uint32_t* listed)
{
    FG_LOOP(l, z.nl())
    {
        const uint32_t c = seg_end[l];
        if (c == 0)
            continue;
        const uint32_t b = atomicAdd(&alloc[0], c);
        seg_begin[l] = b;
        seg_end[l] = b + c;
        cursor[l] = b;
        listed[atomicAdd(&alloc[1], 1u)] = l;
    }
}

__global__ void k_seg_scatter(const unsigned long long* keys, const uint32_t* count, uint32_t* cursor, uint32_t* slots)
{
    FG_LOOP(t, *count)
    {
        const unsigned long long k = keys[t];
        slots[atomicAdd(&cursor[uint32_t(k >> 32)], 1u)] = uint32_t(k);
    }
}

// After the entries of range [b, e) are sorted in slots: memory indices and
// the split (scan order visits memory columns >= cols/2 first: the range is
// [high ..., low ...], split at the first low entry).
__device__ __forceinline__ void seg_finish_warp(const uint32_t* slots, uint32_t b, uint32_t e, const uint32_t* fm,
    uint32_t split_m, uint32_t* vals, uint32_t* split_out)
{
    const int lane = threadIdx.x & 31;
    uint32_t high = 0;
    for (uint32_t t = b + lane; t < e; t += 32) {
        const uint32_t m = fm[slots[t]];
        vals[t] = m;
        high += m >= split_m ? 1u : 0u;
    }
    for (int o = 16; o > 0; o >>= 1)
        high += __shfl_xor_sync(0xffffffffu, high, o);
    if (lane == 0)
        *split_out = b + high;
}

__global__ void __launch_bounds__(256) k_seg_sort(const uint32_t* listed, const uint32_t* nlisted,
    const uint32_t* seg_begin, const uint32_t* seg_end, uint32_t* slots, const uint32_t* fm, uint32_t split_m,
    uint32_t* vals, uint32_t* seg_split, uint32_t* big, uint32_t* nbig)
{
    __shared__ uint32_t buf[8][SEG_WARP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    uint32_t* wb = buf[warp];
    for (uint32_t q = blockIdx.x * (blockDim.x >> 5) + warp, nq = *nlisted; q < nq; q += nwarps) {
        const uint32_t l = listed[q];
        const uint32_t b = seg_begin[l], e = seg_end[l], c = e - b;
        if (c == 0)
            continue;
        if (c > uint32_t(SEG_WARP)) {
            if (lane == 0)
                big[atomicAdd(nbig, 1u)] = l;
            continue;
        }
        if (c <= 32) {
            uint32_t v = uint32_t(lane) < c ? slots[b + lane] : 0xffffffffu;
            for (int k = 2; k <= 32; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const uint32_t o = __shfl_xor_sync(0xffffffffu, v, j);
                    const bool up = (lane & k) == 0, lower = (lane & j) == 0;
                    v = (lower == up) ? min(v, o) : max(v, o);
                }
            if (uint32_t(lane) < c)
                slots[b + lane] = v;
        } else {
            uint32_t p2 = 64;
            while (p2 < c)
                p2 <<= 1;
            for (uint32_t t = lane; t < p2; t += 32)
                wb[t] = t < c ? slots[b + t] : 0xffffffffu;
            __syncwarp();
            for (uint32_t k = 2; k <= p2; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t q = lane; q < (p2 >> 1); q += 32) {
                        const uint32_t lo = 2 * q - (q & (j - 1)), hi = lo + j;
                        const uint32_t x = wb[lo], y = wb[hi];
                        if ((x > y) == ((lo & k) == 0)) {
                            wb[lo] = y;
                            wb[hi] = x;
                        }
                    }
                    __syncwarp();
                }
            for (uint32_t t = lane; t < c; t += 32)
                slots[b + t] = wb[t];
            __syncwarp();
        }
        seg_finish_warp(slots, b, e, fm, split_m, vals, &seg_split[l]);
    }
}

// The ranges above SEG_WARP entries: one block each, up to SEG_BIG entries in
// dynamic shared memory; larger ones set *overflow (the host sorts all the
// entries with the multi-block sort instead).
__global__ void __launch_bounds__(1024) k_seg_sort_big(const uint32_t* seg_begin, const uint32_t* seg_end,
    uint32_t* slots, const uint32_t* fm, uint32_t split_m, uint32_t* vals, uint32_t* seg_split, const uint32_t* big,
    const uint32_t* nbig, uint32_t* overflow)
{
    extern __shared__ uint32_t sb[]; // SEG_BIG
    __shared__ uint32_t whigh[32];
    const uint32_t n = *nbig;
    for (uint32_t q = blockIdx.x; q < n; q += gridDim.x) {
        const uint32_t l = big[q];
        const uint32_t b = seg_begin[l], e = seg_end[l], c = e - b;
        if (c > uint32_t(SEG_BIG)) {
            if (threadIdx.x == 0)
                *overflow = 1u;
            continue;
        }
        uint32_t p2 = 2 * SEG_WARP;
        while (p2 < c)
            p2 <<= 1;
        for (uint32_t t = threadIdx.x; t < p2; t += blockDim.x)
            sb[t] = t < c ? slots[b + t] : 0xffffffffu;
        __syncthreads();
        for (uint32_t k = 2; k <= p2; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t r = threadIdx.x; r < (p2 >> 1); r += blockDim.x) {
                    const uint32_t lo = 2 * r - (r & (j - 1)), hi = lo + j;
                    const uint32_t x = sb[lo], y = sb[hi];
                    if ((x > y) == ((lo & k) == 0)) {
                        sb[lo] = y;
                        sb[hi] = x;
                    }
                }
                __syncthreads();
            }
        uint32_t high = 0;
        for (uint32_t t = threadIdx.x; t < c; t += blockDim.x) {
            const uint32_t i = sb[t];
            slots[b + t] = i;
            const uint32_t m = fm[i];
            vals[b + t] = m;
            high += m >= split_m ? 1u : 0u;
        }
        for (int o = 16; o > 0; o >>= 1)
            high += __shfl_xor_sync(0xffffffffu, high, o);
        if ((threadIdx.x & 31) == 0)
            whigh[threadIdx.x >> 5] = high;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t h = 0;
            for (int w = 0; w < int(blockDim.x >> 5); w++)
                h += whigh[w];
            seg_split[l] = b + h;
        }
        __syncthreads();
    }
}

// List position of the j-th pixel (memory order) of segment [b, e) split at sp.
__device__ __forceinline__ uint32_t seg_at(uint32_t b, uint32_t sp, uint32_t e, uint32_t j)
{
    return j < e - sp ? sp + j : b + (j - (e - sp));
}

// One thread per label: ordered sums over its pixels, with explicitly
// rounded operations (no FMA contraction), so the sums are bit-identical to
// the reference's.  mom: 6 doubles per label code: sum x v, y v, x^2 v,
// y^2 v, x y v, v (display coordinates).
template <typename T>
__global__ void k_label_sums(FgSizes z, const T* img, int rows, int cols, const uint32_t* vals,
    const uint32_t* seg_begin, const uint32_t* seg_end, const uint32_t* seg_split, double* mom, int* ns)
{
    FG_LOOP(l, z.nl())
    {
        const uint32_t b = seg_begin[l], e = seg_end[l], sp = seg_split[l], len = e - b;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0, a5 = 0.0;
        const int vs = rows / 2, hs = cols / 2;
        auto add = [&](uint32_t m, double val) {
            const int c = int(m / uint32_t(rows)), r = int(m - uint32_t(c) * uint32_t(rows));
            const double y = r < vs ? double(r + vs) : double(r - vs);
            const double x = c < hs ? double(c + hs) : double(c - hs);
            const double xb = __dmul_rn(x, val), yb = __dmul_rn(y, val);
            a0 = __dadd_rn(a0, xb);
            a1 = __dadd_rn(a1, yb);
            a2 = __dadd_rn(a2, __dmul_rn(xb, x));
            a3 = __dadd_rn(a3, __dmul_rn(yb, y));
            a4 = __dadd_rn(a4, __dmul_rn(xb, y));
            a5 = __dadd_rn(a5, val);
        };
        // four pixels' loads in flight, then their sums in order
        uint32_t j = 0;
        for (; j + 4 <= len; j += 4) {
            uint32_t m[4];
            double val[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
                m[q] = vals[seg_at(b, sp, e, j + q)];
#pragma unroll
            for (int q = 0; q < 4; q++)
                val[q] = ld(img, m[q]);
#pragma unroll
            for (int q = 0; q < 4; q++)
                add(m[q], val[q]);
        }
        for (; j < len; j++) {
            const uint32_t m = vals[seg_at(b, sp, e, j)];
            add(m, ld(img, m));
        }
        double* mo = mom + 6 * size_t(l);
        mo[0] = a0;
        mo[1] = a1;
        mo[2] = a2;
        mo[3] = a3;
        mo[4] = a4;
        mo[5] = a5;
        ns[l] = int(len);
    }
}


struct IslandRaw {
    int32_t label;
    int32_t num_samples;
    double extremum_val;
    long long extremum_idx;
    double mom[6];
};

// One thread per label (positives [0, np), negatives [np, np + nn)): the
// extremum and its first index (PACKED: unpacked from the single-precision
// keys), the valid-label count (extremum beyond the detection threshold,
// sourcefind.cpp:380-456) and, for valid labels of at least min_area
// pixels, the island record appended at an atomic cursor (the host orders
// the records by label).
template <bool PACKED>
__global__ void k_islands(FgSizes z, const SfStats* st, const unsigned long long* ext,
    const unsigned long long* eidx, const int* ns, const double* mom, int min_area, uint32_t* nvalid, uint32_t* nisl,
    IslandRaw* out)
{
    const int np = z.np();
    FG_LOOP(ut, z.nl())
    {
        const int t = int(ut);
        const bool pos = t < np;
        unsigned long long key, idx;
        bool valid;
        if constexpr (PACKED) {
            const uint32_t hi = uint32_t(ext[t] >> 32), lo = uint32_t(ext[t]);
            valid = hi != (pos ? st->fpos : st->fneg);
            key = okey(double(fkey32_inv(hi)));
            idx = pos ? (unsigned long long)(0xffffffffu - lo) : (unsigned long long)lo;
        } else {
            key = ext[t];
            idx = eidx[t];
            valid = pos ? key > st->kpos : key < st->kneg;
        }
        if (!valid)
            continue;
        atomicAdd(nvalid, 1u);
        if (ns[t] < min_area)
            continue;
        IslandRaw r;
        const int i = pos ? t : t - np;
        r.label = pos ? (i + 1) : -(i + 1);
        r.num_samples = ns[t];
        r.extremum_val = okey_inv(key);
        r.extremum_idx = (long long)idx;
        for (int q = 0; q < 6; q++)
            r.mom[q] = mom[6 * size_t(t) + q];
        out[atomicAdd(nisl, 1u)] = r;
    }
}

// ---------------------------------------------------------------- 2-D Gaussian fit
//
// Least-squares fit of A exp(-(a dx^2 + b dx dy + c dy^2)) to the pixels of
// each island (the model and residual of GaussianResidual,
// src/stp/sourcefind/fitting.h:183-210; a, b, c from the standard deviations
// and theta as there), starting from the moments fit
// (sourcefind.cpp:719-760).  The reference minimises with Ceres; here a
// Levenberg-Marquardt iteration with analytic derivatives: one warp per
// island, lanes over the island's pixels, the 6x6 normal equations reduced
// with shuffles and solved by every lane (Cholesky).
constexpr int FIT_MAX_ITER = 100;

struct GaussTerms {
    double a, b, c, da_dsx, db_dsx, dc_dsx, da_dsy, db_dsy, dc_dsy, da_dt, db_dt, dc_dt;
};

__device__ __forceinline__ GaussTerms gauss_terms(const double* p)
{
    GaussTerms g;
    const double ct = cos(p[5]), st = sin(p[5]), s2t = sin(2.0 * p[5]), c2t = cos(2.0 * p[5]);
    const double ct2 = ct * ct, st2 = st * st;
    const double ix2 = 1.0 / (p[3] * p[3]), iy2 = 1.0 / (p[4] * p[4]);
    const double ix3 = ix2 / p[3], iy3 = iy2 / p[4];
    g.a = 0.5 * (ct2 * ix2 + st2 * iy2);
    g.b = 0.5 * (s2t * ix2 - s2t * iy2);
    g.c = 0.5 * (st2 * ix2 + ct2 * iy2);
    g.da_dsx = -ct2 * ix3;
    g.db_dsx = -s2t * ix3;
    g.dc_dsx = -st2 * ix3;
    g.da_dsy = -st2 * iy3;
    g.db_dsy = s2t * iy3;
    g.dc_dsy = -ct2 * iy3;
    g.da_dt = 0.5 * s2t * (iy2 - ix2);
    g.db_dt = c2t * (ix2 - iy2);
    g.dc_dt = 0.5 * s2t * (ix2 - iy2);
    return g;
}

// Sum over the warp, broadcast from lane 0 so that every lane holds the same
// bits (the butterfly adds in a different order on each lane).
__device__ __forceinline__ double warp_sum_bcast(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Cholesky solve of the 6x6 SPD system m x = r (m: 21 packed lower entries).
__device__ __forceinline__ bool solve6(const double* m, const double* r, double* x)
{
    double L[6][6];
    int t = 0;
    for (int i = 0; i < 6; i++)
        for (int j = 0; j <= i; j++)
            L[i][j] = m[t++];
    for (int j = 0; j < 6; j++) {
        double d = L[j][j];
        for (int k = 0; k < j; k++)
            d -= L[j][k] * L[j][k];
        if (!(d > 0.0))
            return false;
        d = sqrt(d);
        L[j][j] = d;
        for (int i = j + 1; i < 6; i++) {
            double v = L[i][j];
            for (int k = 0; k < j; k++)
                v -= L[i][k] * L[j][k];
            L[i][j] = v / d;
        }
    }
    double y[6];
    for (int i = 0; i < 6; i++) {
        double v = r[i];
        for (int k = 0; k < i; k++)
            v -= L[i][k] * y[k];
        y[i] = v / L[i][i];
    }
    for (int i = 5; i >= 0; i--) {
        double v = y[i];
        for (int k = i + 1; k < 6; k++)
            v -= L[k][i] * x[k];
        x[i] = v / L[i][i];
    }
    return true;
}

// pix[sb[key] .. se[key]) are the island's pixels (memory indices of the
// column-major rows x cols image), in memory order from sp[key] (seg_at);
// x, y are display coordinates (the image is unshifted: display = memory
// index shifted by half, sourcefind.cpp:230-245).
template <typename T>
__global__ void __launch_bounds__(32) k_gauss_fit(const T* __restrict__ img, int rows, int cols,
    const uint32_t* __restrict__ pix, const uint32_t* __restrict__ sb, const uint32_t* __restrict__ se,
    const uint32_t* __restrict__ sp, const int* __restrict__ keys, const double* __restrict__ init, int nis,
    double* outp, int* iters)
{
    const int isl = blockIdx.x;
    if (isl >= nis)
        return;
    const int lane = threadIdx.x;
    const int key = keys[isl];
    const uint32_t b = sb[key], e = se[key], split = sp[key];
    const int hs = cols / 2, vs = rows / 2;
    double p[6];
    for (int k = 0; k < 6; k++)
        p[k] = init[6 * isl + k];

    // cost (and optionally the normal equations) at parameters q
    auto pass = [&](const double* q, bool normal, double* JtJ, double* Jtr) -> double {
        const GaussTerms g = gauss_terms(q);
        double cost = 0.0;
        double jj[21], jr[6];
        if (normal) {
            for (int k = 0; k < 21; k++)
                jj[k] = 0.0;
            for (int k = 0; k < 6; k++)
                jr[k] = 0.0;
        }
        for (uint32_t j = lane; j < e - b; j += 32) {
            const uint32_t m = pix[seg_at(b, split, e, j)];
            const int rm = int(m % uint32_t(rows)), cm = int(m / uint32_t(rows));
            const double x = double(cm < hs ? cm + hs : cm - hs);
            const double y = double(rm < vs ? rm + vs : rm - vs);
            const double dx = x - q[1], dy = y - q[2];
            const double quad = g.a * dx * dx + g.b * dx * dy + g.c * dy * dy;
            const double ex = exp(-quad);
            const double r = q[0] * ex - double(img[m]);
            cost += r * r;
            if (normal) {
                const double ae = q[0] * ex;
                double J[6];
                J[0] = ex;
                J[1] = ae * (2.0 * g.a * dx + g.b * dy);
                J[2] = ae * (g.b * dx + 2.0 * g.c * dy);
                J[3] = -ae * (g.da_dsx * dx * dx + g.db_dsx * dx * dy + g.dc_dsx * dy * dy);
                J[4] = -ae * (g.da_dsy * dx * dx + g.db_dsy * dx * dy + g.dc_dsy * dy * dy);
                J[5] = -ae * (g.da_dt * dx * dx + g.db_dt * dx * dy + g.dc_dt * dy * dy);
                int u = 0;
                for (int i = 0; i < 6; i++) {
                    jr[i] += J[i] * r;
                    for (int j = 0; j <= i; j++)
                        jj[u++] += J[i] * J[j];
                }
            }
        }
        if (normal) {
            for (int k = 0; k < 21; k++)
                JtJ[k] = warp_sum_bcast(jj[k]);
            for (int k = 0; k < 6; k++)
                Jtr[k] = warp_sum_bcast(jr[k]);
        }
        return warp_sum_bcast(cost);
    };

    double JtJ[21], Jtr[6];
    double cost = pass(p, true, JtJ, Jtr);
    double lambda = 1e-3;
    int it = 0;
    while (it < FIT_MAX_ITER) {
        it++;
        // (J^T J + lambda D) delta = -J^T r, D = diag(J^T J) floored at 1e-12 of its
        // largest entry (a parameter the residuals do not depend on, such as
        // theta of a circular Gaussian, then gets a zero step)
        double m[21], rhs[6], d[6], q[6];
        double dmax = 0.0;
        for (int i = 0; i < 6; i++)
            dmax = fmax(dmax, JtJ[i * (i + 1) / 2 + i]);
        int u = 0;
        for (int i = 0; i < 6; i++) {
            rhs[i] = -Jtr[i];
            for (int j = 0; j <= i; j++, u++)
                m[u] = (i == j) ? JtJ[u] + lambda * fmax(JtJ[u], 1e-12 * dmax + 1e-300) : JtJ[u];
        }
        bool ok = solve6(m, rhs, d);
        double cnew = 0.0;
        if (ok) {
            for (int k = 0; k < 6; k++)
                q[k] = p[k] + d[k];
            ok = q[3] != 0.0 && q[4] != 0.0;
        }
        if (ok) {
            double dummy1[21], dummy2[6];
            cnew = pass(q, false, dummy1, dummy2);
            ok = cnew == cnew && cnew < cost; // NaN-safe
        }
        if (ok) {
            double step = 0.0;
            for (int k = 0; k < 6; k++)
                step = fmax(step, fabs(d[k]) / (fabs(p[k]) + 1e-10));
            const bool small = (cost - cnew) <= 1e-12 * cost || step <= 1e-10;
            for (int k = 0; k < 6; k++)
                p[k] = q[k];
            cost = pass(p, true, JtJ, Jtr);
            lambda = fmax(lambda * 0.1, 1e-15);
            if (small)
                break;
        } else {
            lambda *= 10.0;
            if (lambda > 1e16)
                break;
        }
    }
    if (lane == 0) {
        for (int k = 0; k < 6; k++)
            outp[6 * isl + k] = p[k];
        iters[isl] = it;
    }
}

} // namespace stpgpu
