// Device kernels of the snapshot imager.
//
// Pipeline (one snapshot):
//   k_prepass      uvw -> pixel scaling, half-plane conversion, rint split,
//                  bounds check, uv shift, oversampled index  (gridder.h:369-504)
//   [W-proj]       |w| sort (CUB), plane boundaries/averages, FP64 W-kernels
//   k_count_tiles  footprint -> uv tiles it overlaps (counting pass)
//   k_scan_*       tile offsets
//   k_fill_tiles   tile -> item lists
//   k_grid_tiles   one CTA per 32x32 tile of the half-plane grid: all items
//                  whose footprint touches the tile accumulate in shared
//                  memory, then the tile is written once with coalesced
//                  stores (no memset, no global atomics)          (gridder.h:596-994)
//   cuFFT Z2D/C2R  (fft.cpp:45-135)
//   k_normalise    crop + 1/sum + gcf division                    (imager.h:97-150)
#pragma once

#include "common.cuh"

namespace stpgpu {

constexpr int TILE_R = 32; // tile rows (v, the fast grid axis)
constexpr int TILE_C_DEFAULT = 32; // tile columns (u); 16-column tiles are the other tuned shape
constexpr int GRID_THREADS = 256;

enum KMode { KM_SEP = 0, KM_EXACT = 1, KM_WPROJ = 2 };

// Per-visibility record written by the prepass.  flags: bit0 conj(kernel)
// for the original item (w < 0), bit1 conj(kernel) for the mirrored item
// (-w < 0).  The visibility is stored conjugated when the half-plane
// conversion flipped it.  16-byte aligned (32 B single, 48 B double
// precision): a record never straddles a 32-byte sector more than it must,
// and the gridder's random fetch of a record is two or three 16-byte loads.
template <typename R>
struct alignas(16) Item {
    R vr, vi, w;
    int32_t gcx, gcy;
    int16_t cpx, cpy;
    uint16_t plane;
    uint8_t good, flags;
};
static_assert(sizeof(Item<float>) == 32 && sizeof(Item<double>) == 48, "item record sizes");

struct PrepassParams {
    int64_t n;
    const void* vis; // complex128 or complex64
    int vis_c64;
    const double* weights;
    const double* uv; // either uvw (n x 3, lambda) or uv (n x 2, pixels)
    int uv_is_pixels;
    double inv_px; // lambda -> pixel factor when uv_is_pixels == 0
    int N, conv_support, halfplane, shift_uv, kernel_exact, os;
    int keep_w;
    double* frac;      // 2n (exact mode only), may be null
    double* wsum_part; // per-block partial sums of good weights
    unsigned long long* ngood_part;
    double* absw_key; // n |w| (W-proj only), may be null
    double* w_out;    // n half-plane-converted w (W-proj), may be null
    double* wmax_part; // per block: the maximum and the sum of the finite |w| (W-proj), may be null
    uint32_t* iota;    // n identity permutation (W-proj), may be null
};

template <typename R>
__global__ void k_prepass(PrepassParams p, Item<R>* items)
{
    __shared__ double s_w[GRID_THREADS / 32];
    __shared__ unsigned long long s_n[GRID_THREADS / 32];
    __shared__ double s_m[GRID_THREADS / 32], s_a[GRID_THREADS / 32];
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    double wgood = 0.0, wmax = 0.0, wabs = 0.0;
    unsigned long long ngood = 0;
    if (i < p.n) {
        double u, v, w = 0.0;
        if (p.uv_is_pixels) {
            u = p.uv[i];
            v = p.uv[p.n + i];
            if (p.keep_w)
                w = p.uv[2 * p.n + i];
        } else {
            u = p.uv[i] * p.inv_px;
            v = p.uv[p.n + i] * p.inv_px;
            w = p.uv[2 * p.n + i];
        }
        double vr, vi;
        if (p.vis_c64) {
            float2 t = reinterpret_cast<const float2*>(p.vis)[i];
            vr = t.x;
            vi = t.y;
        } else {
            double2 t = reinterpret_cast<const double2*>(p.vis)[i];
            vr = t.x;
            vi = t.y;
        }
        const double wt = p.weights[i];
        int good = 1;
        const int S = p.conv_support;
        if (p.halfplane) {
            if (v < 0.0) {
                if (v > -(S + 1))
                    good = 2;
                u *= -1;
                v *= -1;
                w *= -1;
                vi = -vi;
            } else if (v < (S + 1)) {
                good = 2;
            }
        }
        const int half = p.N / 2;
        bool finite = isfinite(u) && isfinite(v);
        double ru = rint(u), rv = rint(v);
        // int(rint(x)) with the out-of-range behaviour of x86 (INT_MIN) kept
        // for the bounds check: such centres are always out of bounds.
        long long vx = (finite && fabs(ru) < 1.0e9) ? (long long)ru : (long long)INT32_MIN;
        long long vy = (finite && fabs(rv) < 1.0e9) ? (long long)rv : (long long)INT32_MIN;
        double fx = u - double(vx), fy = v - double(vy);
        long long kx = vx + half, ky = vy + half;
        if (!finite || (kx - S) <= 0 || (ky - S) <= 0 || (kx + S) >= p.N || (ky + S) >= p.N)
            good = 0;
        if (p.shift_uv) {
            kx = kx < half ? kx + half : kx - half;
            ky = ky < half ? ky + half : ky - half;
        }
        int cpx = 0, cpy = 0;
        if (!p.kernel_exact) {
            const int rmax = p.os / 2;
            int ox = int(rint(fx * p.os)), oy = int(rint(fy * p.os));
            ox = ox > rmax ? rmax : (ox < -rmax ? -rmax : ox);
            oy = oy > rmax ? rmax : (oy < -rmax ? -rmax : oy);
            cpx = ox + rmax;
            cpy = oy + rmax;
        }
        if (p.frac) {
            p.frac[i] = fx;
            p.frac[p.n + i] = fy;
        }
        if (p.absw_key)
            p.absw_key[i] = fabs(w);
        if (fabs(w) <= 1.7976931348623157e308) { // finite
            wmax = fabs(w);
            wabs = fabs(w);
        }
        if (p.iota)
            p.iota[i] = uint32_t(i);
        if (p.w_out)
            p.w_out[i] = w;
        Item<R> it;
        it.vr = R(vr);
        it.vi = R(vi);
        it.w = R(wt);
        it.gcx = good ? int32_t(kx) : 0;
        it.gcy = good ? int32_t(ky) : 0;
        it.cpx = int16_t(cpx);
        it.cpy = int16_t(cpy);
        it.plane = 0;
        it.good = uint8_t(good);
        it.flags = uint8_t((w < 0.0 ? 1 : 0) | (-w < 0.0 ? 2 : 0));
        items[i] = it;
        if (good) {
            wgood = wt;
            ngood = 1;
        }
    }
    // deterministic block partial sums
    for (int o = 16; o > 0; o >>= 1) {
        wgood += __shfl_down_sync(0xffffffffu, wgood, o);
        ngood += __shfl_down_sync(0xffffffffu, ngood, o);
        wmax = fmax(wmax, __shfl_down_sync(0xffffffffu, wmax, o));
        wabs += __shfl_down_sync(0xffffffffu, wabs, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_w[threadIdx.x >> 5] = wgood;
        s_n[threadIdx.x >> 5] = ngood;
        s_m[threadIdx.x >> 5] = wmax;
        s_a[threadIdx.x >> 5] = wabs;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0, m = 0.0, a = 0.0;
        unsigned long long c = 0;
        for (int k = 0; k < int(blockDim.x >> 5); k++) {
            t += s_w[k];
            c += s_n[k];
            m = fmax(m, s_m[k]);
            a += s_a[k];
        }
        p.wsum_part[blockIdx.x] = t;
        p.ngood_part[blockIdx.x] = c;
        if (p.wmax_part) {
            p.wmax_part[2 * blockIdx.x] = m;
            p.wmax_part[2 * blockIdx.x + 1] = a;
        }
    }
}

// Sum of block partials in a fixed order (one block).  out[0] = 2 * sum
// (the half-plane doubling of gridder.h:423), out_n[0] = count; with mpart,
// out[1] = the largest finite |w| and out[2] = the sum of the finite |w|.
__global__ void k_finish_wsum(const double* part, const unsigned long long* npart, const double* mpart, int nb,
    double* out, unsigned long long* out_n)
{
    __shared__ double s[1024];
    __shared__ unsigned long long sn[1024];
    __shared__ double sm[1024], sa[1024];
    double t = 0.0, m = 0.0, a = 0.0;
    unsigned long long c = 0;
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        t += part[k];
        c += npart[k];
        if (mpart) {
            m = fmax(m, mpart[2 * k]);
            a += mpart[2 * k + 1];
        }
    }
    s[threadIdx.x] = t;
    sn[threadIdx.x] = c;
    sm[threadIdx.x] = m;
    sa[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s[threadIdx.x] += s[threadIdx.x + o];
            sn[threadIdx.x] += sn[threadIdx.x + o];
            sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
            sa[threadIdx.x] += sa[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s[0] * 2.0;
        out_n[0] = sn[0];
        if (mpart) {
            out[1] = sm[0];
            out[2] = sa[0];
        }
    }
}

// Sort keys of |w| for the W-plane order, 24 bits, monotone in |w| (|a| <=
// |b| implies key(a) <= key(b)), so that a stable sort of the keys followed
// by k_fix_runs (runs of equal keys re-sorted by the full |w| bits, NaN after
// every number) gives the order of the IEEE bits of |w|.  With x = |w| /
// wmax (wmax = total[1], the largest finite |w|), two encodings, chosen by
// how far the mean |w| (total[2] / n) sits below wmax so that runs of equal
// keys stay short:
//  * spread |w| (mean >= wmax / 16): floor(sqrt(x) (2^24 - 2)), resolution
//    2^-24 in sqrt(x) (about 8 % of the headline snapshot's keys in runs);
//  * |w| concentrated far below wmax: x rounded down to single precision and
//    raised to at least 2^-31, key = (bits(x) - bits(2^-31)) >> 4 (the 32
//    exponents from 2^-31 to 1 and 19 mantissa bits: relative resolution
//    2^-19 at every scale).
// Non-finite |w| (NaN included) take 2^24 - 1, above every finite key.
struct WKey {
    double wmax, r;
    bool spread;
    __device__ WKey(const double* total, int64_t n)
    {
        wmax = total[1];
        r = wmax > 0.0 ? 1.0 / wmax : 0.0;
        spread = wmax > 0.0 && total[2] >= wmax * 0.0625 * double(n);
    }
    __device__ __forceinline__ uint32_t operator()(double a) const
    {
        uint32_t k = 0xFFFFFFu;
        if (a <= wmax) {
            if (spread) {
                const double q = __dsqrt_rn(a * r) * 16777214.0;
                k = q < 16777214.0 ? uint32_t(q) : 16777214u;
            } else {
                const float x = fmaxf(__double2float_rd(a * r), 0x1p-31f);
                k = (__float_as_uint(x) - 0x30000000u) >> 4;
            }
        }
        return k;
    }
};

__global__ void k_wkey24(const double* __restrict__ absw, int64_t n, const double* total, uint32_t* __restrict__ key)
{
    const WKey kf(total, n);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        key[i] = kf(absw[i]);
}

// Zeroes up to four ranges of 32-bit words (one launch instead of several
// memset nodes in a captured call).
struct ZeroRanges {
    uint32_t* p[4];
    int64_t n[4];
};
__global__ void k_zero_ranges(ZeroRanges z)
{
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x, st = int64_t(gridDim.x) * blockDim.x;
#pragma unroll
    for (int r = 0; r < 4; r++)
        if (z.p[r])
            for (int64_t i = t; i < z.n[r]; i += st)
                z.p[r][i] = 0;
}

// ---------------------------------------------------------------- footprint segments

// Footprint index mapping (gridder.h:645-667 columns/rows, :970-983 exact).
// Column tap j of a kernel whose left edge is cb lands in grid column
// cb + j wrapped once into [0, N).  Row tap i lands in cb-style wrapped row
// rb + i, except that negative rows are skipped by the oversampled gridder
// and wrapped by the exact one; rows >= `rows` (half plane) are dropped.
// Returns -1 when the tap is not gridded.
__device__ __forceinline__ int map_col(int raw, int N)
{
    return raw < 0 ? raw + N : (raw >= N ? raw - N : raw);
}
__device__ __forceinline__ int map_row(int raw, int N, int rows, bool wrap_neg)
{
    if (raw < 0) {
        if (!wrap_neg)
            return -1;
        raw += N;
    } else if (raw >= N) {
        raw -= N;
    }
    return raw < rows ? raw : -1;
}

constexpr int kRankSlots = 4; // tiles per (item, mirror) whose list slots the count pass keeps

// One (entry, tile) pair of the binning, decoded for the staged gridder
// (grid_tile_recs): the entry's footprint clipped to the tile, the weighted
// visibility and the kernel-table offset of the window's first tap.  The
// fill pass writes these records contiguously in tile order, so a tile's
// entries are one contiguous byte range that the gridder copies into shared
// memory with bulk (TMA) copies.  16 B in single precision, 32 B in double.
//   geom: row0 (5 bits, local row of the window's first tap), col0 (5 bits),
//         nrows (6 bits, 1..32), ncols (6 bits), conj (1 bit, W-kernel
//         conjugated), K (8 bits, kernel width; the row stride of W-kernels)
//   koff: W-projection: index of tap (ilo, jlo) in the expanded kernel
//         tables; separable: (cpy*K + ilo) << 16 | (cpx*K + jlo)
template <typename R>
struct alignas(16) TapRec {
    R vr, vi;
    uint32_t koff;
    uint32_t geom;
};
static_assert(sizeof(TapRec<float>) == 16 && sizeof(TapRec<double>) == 32, "tile record sizes");

__host__ __device__ __forceinline__ uint32_t rec_geom(int row0, int col0, int nrows, int ncols, int conj, int K)
{
    return uint32_t(row0) | (uint32_t(col0) << 5) | (uint32_t(nrows) << 10) | (uint32_t(ncols) << 16)
        | (uint32_t(conj & 1) << 22) | (uint32_t(K) << 23);
}

struct BinParams {
    int N, image_rows, tiles_r, tiles_c;
    int tile_c;              // tile width in grid columns (TILE_R rows per tile)
    int support;             // non-W-proj support
    const int* plane_support; // W-proj truncated support per plane (nullable)
    const uint16_t* plane16;  // W-proj without the |w| sort: plane of each item (input order), else null
    const uint8_t* ts_of;     // A-projection: time step per visibility (nullable)
    int ntimesteps;           // planes are indexed plane * ntimesteps + step
    int exact;               // rows wrap negative (exact gridder)
    int64_t n;
    uint32_t* tile_count;
    const uint32_t* tile_off;
    uint32_t* tile_cursor;
    uint32_t* ranks;          // nullable: [kRankSlots][2][n] list slots taken by the count pass
    uint32_t* rank_overflow;  // set when some (item, mirror) touched more than kRankSlots tiles
    uint32_t* list;
    uint64_t list_capacity;
    unsigned int* err;
};

template <typename R>
__device__ __forceinline__ void item_centre(const Item<R>& it, int mir, int N, int& cx, int& cy)
{
    cx = mir ? N - it.gcx : it.gcx;
    cy = mir ? N - it.gcy : it.gcy;
}

// Tiles overlapped by one item: calls f(tile) once per distinct tile.  The
// footprint's raw rows [rb, rb+K) and columns [cb, cb+K) are split into the
// segments that map_row / map_col send to distinct grid ranges (in place,
// wrapped from >= N, and for the exact gridder wrapped from < 0; rows at or
// beyond the half plane dropped); each segment becomes a range of tile
// indices, overlapping ranges are merged, and the tiles of the row ranges x
// column ranges are visited once each.
struct TileRanges {
    int lo[3], hi[3];
    int n;
    __device__ __forceinline__ void add(int l, int h)
    {
        if (l > h)
            return;
        for (int k = 0; k < n; k++) {
            if (l <= hi[k] + 1 && h >= lo[k] - 1) { // overlapping or adjacent: merge
                lo[k] = min(lo[k], l);
                hi[k] = max(hi[k], h);
                return;
            }
        }
        lo[n] = l;
        hi[n] = h;
        n++;
    }
    // merge ranges that a later add made overlap
    __device__ __forceinline__ void merge()
    {
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                if (lo[b] <= hi[a] + 1 && hi[b] >= lo[a] - 1) {
                    lo[a] = min(lo[a], lo[b]);
                    hi[a] = max(hi[a], hi[b]);
                    lo[b] = lo[n - 1];
                    hi[b] = hi[n - 1];
                    n--;
                    b = a; // restart the scan of a
                }
    }
};

template <typename R, typename F>
__device__ __forceinline__ void for_item_tiles(const Item<R>& it, int mir, int S, const BinParams& p, F f)
{
    const int K = 2 * S + 1;
    int cx, cy;
    item_centre(it, mir, p.N, cx, cy);
    const int N = p.N, rows_max = p.image_rows - 1;
    const int a = cy - S, b = cy - S + K - 1; // raw rows
    {
        // common case: the footprint wraps on neither axis, so it covers one
        // range of tile rows and one of tile columns (tile sizes are powers
        // of two; every index here is non-negative)
        const int c = cx - S, d = cx - S + K - 1;
        if (a >= 0 && b < N && c >= 0 && d < N) {
            const int h = min(b, rows_max);
            if (a > h)
                return;
            const int cshift = p.tile_c == 32 ? 5 : (p.tile_c == 16 ? 4 : 3);
            for (int t_r = a / TILE_R; t_r <= h / TILE_R; t_r++)
                for (int t_c = c >> cshift; t_c <= (d >> cshift); t_c++)
                    f(uint32_t(t_c) * uint32_t(p.tiles_r) + uint32_t(t_r));
            return;
        }
    }
    TileRanges tr;
    tr.n = 0;
    {
        const int l = max(a, 0), h = min(min(b, N - 1), rows_max);
        if (l <= h)
            tr.add(l / TILE_R, h / TILE_R);
    }
    if (b >= N) {
        const int l = max(a, N) - N, h = min(b - N, rows_max);
        if (l <= h)
            tr.add(l / TILE_R, h / TILE_R);
    }
    if (p.exact && a < 0) {
        const int l = a + N, h = min(min(b, -1) + N, rows_max);
        if (l <= h)
            tr.add(l / TILE_R, h / TILE_R);
    }
    if (tr.n == 0)
        return;
    const int c = cx - S, d = cx - S + K - 1; // raw columns
    TileRanges tc;
    tc.n = 0;
    {
        const int l = max(c, 0), h = min(d, N - 1);
        if (l <= h)
            tc.add(l / p.tile_c, h / p.tile_c);
    }
    if (c < 0)
        tc.add((c + N) / p.tile_c, (min(d, -1) + N) / p.tile_c);
    if (d >= N)
        tc.add((max(c, N) - N) / p.tile_c, (d - N) / p.tile_c);
    tr.merge();
    tc.merge();
    for (int r = 0; r < tr.n; r++)
        for (int t_r = tr.lo[r]; t_r <= tr.hi[r]; t_r++)
            for (int q = 0; q < tc.n; q++)
                for (int t_c = tc.lo[q]; t_c <= tc.hi[q]; t_c++)
                    f(uint32_t(t_c) * uint32_t(p.tiles_r) + uint32_t(t_r));
}

// W-plane of sorted position k: the last plane whose first position <= k.
__device__ __forceinline__ int plane_of(const int64_t* first, int P, int64_t k)
{
    int lo = 0, hi = P - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (first[mid] <= k)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// With W-projection (`order` = the |w| permutation, `first` = plane starts)
// `items` is already permuted into |w| order (item k is sorted position k);
// each item takes the plane of its position, which the fill pass records in
// the item for the gridder (order[k] is the item's input index, used for
// per-visibility inputs such as the A-projection time step).
template <typename R>
__global__ void k_count_tiles(BinParams p, const Item<R>* items, const uint32_t* order, const int64_t* first, int P)
{
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= p.n)
        return;
    const Item<R> it = items[k];
    if (!it.good)
        return;
    int S = p.support;
    if (p.plane16) {
        S = p.plane_support[p.plane16[k]];
    } else if (order) {
        int plane = plane_of(first, P, k);
        if (p.ts_of)
            plane = plane * p.ntimesteps + p.ts_of[order[k]];
        S = p.plane_support[plane];
    }
    for (int mir = 0; mir < int(it.good); mir++) {
        // the count's atomic returns the entry's slot in the tile list; up to
        // kRankSlots of them per (item, mirror) are kept for the fill pass
        int q = 0;
        for_item_tiles(it, mir, S, p, [&](uint32_t t) {
            const uint32_t r = atomicAdd(&p.tile_count[t], 1u);
            if (p.ranks) {
                if (q < kRankSlots)
                    p.ranks[size_t(q * 2 + mir) * size_t(p.n) + size_t(k)] = r; // slot-major: coalesced
                else
                    *p.rank_overflow = 1u;
            }
            q++;
        });
    }
}

// Lists are filled in |w| order for W-projection, so that a warp's items
// mostly share one plane.
template <typename R>
__global__ void k_fill_tiles(BinParams p, Item<R>* items, const uint32_t* order, const int64_t* first, int P)
{
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= p.n)
        return;
    const int64_t i = k;
    const Item<R> it = items[k];
    if (!it.good)
        return;
    int S = p.support;
    if (p.plane16) {
        const int plane = p.plane16[k];
        S = p.plane_support[plane];
        items[k].plane = uint16_t(plane);
    } else if (order) {
        int plane = plane_of(first, P, k);
        if (p.ts_of)
            plane = plane * p.ntimesteps + p.ts_of[order[k]];
        S = p.plane_support[plane];
        items[k].plane = uint16_t(plane);
    }
    // slots from the count pass when every (item, mirror) kept its slots
    // (no footprint with more than kRankSlots tiles), else from cursors
    const bool ranked = p.ranks && *p.rank_overflow == 0u;
    for (int mir = 0; mir < int(it.good); mir++) {
        int q = 0;
        for_item_tiles(it, mir, S, p, [&](uint32_t t) {
            const uint32_t slot = ranked ? p.ranks[size_t(q * 2 + mir) * size_t(p.n) + size_t(k)]
                                         : atomicAdd(&p.tile_cursor[t], 1u);
            q++;
            const uint64_t pos = uint64_t(p.tile_off[t]) + slot;
            if (pos < p.list_capacity)
                p.list[pos] = uint32_t(i) * 2u + uint32_t(mir);
            else
                atomicOr(p.err, 1u);
        });
    }
}

// Exclusive scan of n counts into off[0..n] (single block of 1024 threads,
// n up to a few hundred thousand).  off[n] = total.  Each thread first
// loads 16 elements (16 coalesced rows of 1024), then the rows are scanned
// in order with warp shuffles and one shared-memory step per row.
__device__ __forceinline__ uint32_t scan_block_1024(const uint32_t* cnt, uint32_t* off, int n)
{
    __shared__ uint32_t wsum[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t carry = 0;
    for (int base = 0; base < n; base += 1024 * 16) {
        uint32_t v[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int idx = base + j * 1024 + tid;
            v[j] = idx < n ? cnt[idx] : 0u;
        }
#pragma unroll
        for (int j = 0; j < 16; j++) {
            if (base + j * 1024 >= n)
                break;
            uint32_t x = v[j];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o)
                    x += y;
            }
            if (lane == 31)
                wsum[warp] = x;
            __syncthreads();
            if (warp == 0) {
                uint32_t t = wsum[lane];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
                    if (lane >= o)
                        t += y;
                }
                wsum[lane] = t;
            }
            __syncthreads();
            const int idx = base + j * 1024 + tid;
            if (idx < n)
                off[idx] = carry + (warp ? wsum[warp - 1] : 0u) + x - v[j];
            carry += wsum[31];
            __syncthreads();
        }
    }
    if (tid == 0)
        off[n] = carry;
    return carry;
}

__global__ void __launch_bounds__(1024) k_scan_single(const uint32_t* cnt, uint32_t* off, int n)
{
    scan_block_1024(cnt, off, n);
}

// One such scan per block: row blockIdx.x of cnt and off (row stride
// `stride`); the totals also go to tot[row].
__global__ void __launch_bounds__(1024) k_scan_rows(const uint32_t* cnt, uint32_t* off, int n, int stride, uint32_t* tot)
{
    const uint32_t t = scan_block_1024(cnt + int64_t(blockIdx.x) * stride, off + int64_t(blockIdx.x) * stride, n);
    if (threadIdx.x == 0)
        tot[blockIdx.x] = t;
}

// ---------------------------------------------------------------- accumulators

// Shared-memory cell accumulators.  Each cell is owned by one warp and
// updated with plain read-modify-write (no atomics), so the two-sum
// compensation of FP32C is exact: s + c carries the full sum.
template <typename R, int COMP>
struct Acc;
template <>
struct __align__(16) Acc<double, 0> {
    double2 s;
};
template <>
struct __align__(8) Acc<float, 0> {
    float2 s;
};
template <>
struct __align__(16) Acc<float, 1> {
    float2 s, c;
};

__device__ __forceinline__ void acc_rmw(Acc<double, 0>* a, double re, double im)
{
    double2 v = a->s;
    v.x += re;
    v.y += im;
    a->s = v;
}
__device__ __forceinline__ void acc_rmw(Acc<float, 0>* a, float re, float im)
{
    float2 v = a->s;
    v.x += re;
    v.y += im;
    a->s = v;
}
// Packed single-precision pairs (sm_100 f32x2: one instruction rounds both
// halves, each as its scalar form would).
__device__ __forceinline__ unsigned long long f2_pack(float x, float y)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
    return r;
}
__device__ __forceinline__ float2 f2_unpack(unsigned long long r)
{
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
// FP32C update: t = s + x and Knuth's TwoSum error term
// e = (s - (t - bb)) + (x - bb), bb = t - s, added to c, with explicit
// rounding (no contraction), the real and imaginary parts side by side in
// seven packed adds.  TwoSum is exact whatever the magnitudes: Dekker's
// cheaper Fast2Sum needs |s| >= |x|, which fails throughout a cell whose
// running sum cancels, and there it loses about one rounding of each term
// (enough to move a 256^2 PSWF image by 3e-5 of its peak with the order of
// the updates).
__device__ __forceinline__ void acc_rmw(Acc<float, 1>* a, float re, float im)
{
    const Acc<float, 1> v = *a;
    const unsigned long long s = f2_pack(v.s.x, v.s.y), x = f2_pack(re, im);
    const unsigned long long t = f2_add(s, x);
    const unsigned long long bb = f2_sub(t, s);
    const unsigned long long e = f2_add(f2_sub(s, f2_sub(t, bb)), f2_sub(x, bb));
    Acc<float, 1> w;
    w.s = f2_unpack(t);
    w.c = f2_unpack(f2_add(f2_pack(v.c.x, v.c.y), e));
    *a = w;
}
template <typename R, int COMP>
__device__ __forceinline__ void acc_zero(Acc<R, COMP>* a)
{
    *a = Acc<R, COMP> {};
}
__device__ __forceinline__ double2 acc_value(const Acc<double, 0>& a) { return a.s; }
__device__ __forceinline__ float2 acc_value(const Acc<float, 0>& a) { return a.s; }
__device__ __forceinline__ float2 acc_value(const Acc<float, 1>& a)
{
    return make_float2(__fadd_rn(a.s.x, a.c.x), __fadd_rn(a.s.y, a.c.y));
}

template <typename R>
struct Cplx;
template <>
struct Cplx<double> {
    using T = double2;
};
template <>
struct Cplx<float> {
    using T = float2;
};

// Store of one finished cell: the accumulator's value in the grid's
// precision, or (compensated FP32 into a wide grid) sum + error in double.
template <typename R, int COMP>
__device__ __forceinline__ void cell_store(typename Cplx<R>::T* g, size_t i, const Acc<R, COMP>& a, int wide)
{
    if constexpr (COMP == 1) {
        if (wide) {
            reinterpret_cast<double2*>(g)[i]
                = make_double2(double(a.s.x) + double(a.c.x), double(a.s.y) + double(a.c.y));
            return;
        }
    }
    g[i] = acc_value(a);
}

// ---------------------------------------------------------------- gridder

template <typename R>
struct GridParams {
    int N, image_rows, tiles_r;
    int support, os, cs; // cs = cache size per dimension = (os/2)*2+1
    int exact_wrap;      // exact gridder row wrap
    const Item<R>* items;
    const uint32_t* tile_off;
    const uint32_t* list;
    // KM_SEP: 1-D kernel table [cs][K] (R)
    const R* k1d;
    // KM_EXACT: functor + per-visibility fractions
    int kf;
    double trunc;
    const double* frac;
    int64_t n;
    // KM_WPROJ: per plane the W-kernel quadrant conv[p][l][k] (stride lh,
    // |offsets| index it) and 1/sum(Re) per oversampled offset inv[p][y][x]:
    // the cached kernel of aw_projection.cpp:415-448 is conv * inv.
    const typename Cplx<R>::T* wconv;
    const R* winv;
    int lh;
    const int* plane_support;
    // KM_WPROJ: per plane and oversampled offset pair (cpy, cpx) the K x K
    // cached kernel (conv * inv, tap i*K + j) at wk + wk_off[plane] + (cpy*cs + cpx)*K*K
    const typename Cplx<R>::T* wk;
    const uint32_t* wk_off;
    // staged form (grid_tile_recs): the decoded entries in tile order, and
    // how many the buffer holds
    const TapRec<R>* recs;
    uint64_t rec_cap;
    unsigned int* err; // error flags of the call (staged form: bits 8 and 16)
    typename Cplx<R>::T* grid; // image_rows x N column-major
    typename Cplx<R>::T* beam; // nullable
    // compensated FP32 only: grid and beam hold double2 cells (sum + error
    // term carried into double) for a double-precision c2r transform
    int wide;
};

// One warp per 32x32 tile of the (half-plane) grid.  Lanes take 32 items of
// the tile's list at a time and walk their K x K footprints in lockstep, so
// at every step distinct lanes touch distinct cells unless two items share a
// kernel corner; such items are deferred to a later round (match_any).  The
// tile is zeroed in shared memory, accumulated with plain read-modify-write,
// and stored once with coalesced 512-byte column writes: no memset of the
// grid, no global or shared atomics, and every cell of the grid is written
// exactly once.  (Gridding semantics: gridder.h:596-994.)
// Kernel value of tap (i, j) of the lane's item, times the visibility weight.
template <typename R, int KMODE>
struct TapCtx {
    int K, S, cpx, cpy, os, lh;
    R wt, winv;
    bool conj_k;
    const typename Cplx<R>::T* wconv;
    double fx, fy, ksum;
};

template <typename R, int KMODE>
__device__ __forceinline__ void tap_value(const GridParams<R>& p, const R* tab, const TapCtx<R, KMODE>& t, int i, int j,
    R& kr, R& ki)
{
    if (KMODE == KM_SEP) {
        kr = tab[t.cpy * t.K + i] * tab[t.cpx * t.K + j];
        ki = R(0);
    } else if (KMODE == KM_EXACT) {
        // make_kernel_array (conv_func.h:279-303): outer product / accu
        const double y = kernel_value(p.kf, p.trunc, (double(i) - t.S) - t.fy);
        const double x = kernel_value(p.kf, p.trunc, (double(j) - t.S) - t.fx);
        kr = R((y * x) / t.ksum);
        ki = R(0);
    } else {
        const typename Cplx<R>::T cv = t.wconv[i * t.K + j];
        kr = cv.x;
        ki = t.conj_k ? -cv.y : cv.y;
    }
}

template <typename R, int COMP, int KMODE, bool BEAM, int TILE_C>
__device__ __forceinline__ void grid_tile(const GridParams<R>& p, int tile, unsigned char* smem_raw)
{
    using A = Acc<R, COMP>;
    A* acc = reinterpret_cast<A*>(smem_raw);
    A* bacc = acc + (BEAM ? TILE_R * TILE_C : 0);
    R* tab = reinterpret_cast<R*>(acc + (BEAM ? 2 : 1) * TILE_R * TILE_C);
    const int lane = threadIdx.x;
    // hot scalars in registers (the batch kernel reads p from parameter
    // space with a run-time index, which costs a load per use)
    const int gN = p.N, grows = p.image_rows, gos = p.os, glh = p.lh;
    const int tr = tile % p.tiles_r, tc = tile / p.tiles_r;
    const int r0 = tr * TILE_R, c0 = tc * TILE_C;
    const bool wrap_neg = p.exact_wrap != 0;

    for (int t = lane; t < TILE_R * TILE_C; t += 32) {
        acc_zero(&acc[t]);
        if (BEAM)
            acc_zero(&bacc[t]);
    }
    if (KMODE == KM_SEP) {
        const int K = 2 * p.support + 1;
        for (int t = lane; t < p.cs * K; t += 32)
            tab[t] = p.k1d[t];
    }
    __syncwarp();

    const uint32_t beg = p.tile_off[tile], end = p.tile_off[tile + 1];
    for (uint32_t base = beg; base < end; base += 32) {
        const uint32_t e = base + lane;
        const bool active = e < end;
        TapCtx<R, KMODE> t;
        t.K = 0;
        t.S = 0;
        t.cpx = t.cpy = 0;
        t.os = gos;
        t.lh = glh;
        t.wt = R(0);
        t.winv = R(1);
        t.conj_k = false;
        t.wconv = nullptr;
        t.fx = t.fy = 0.0;
        t.ksum = 1.0;
        R vr = R(0), vim = R(0);
        int rb = 0, cb = 0;
        int cbase = 0, jlo = 0, jhi = 0;
        bool cwrap = false;
        unsigned long long key = ~0ull;
        if (active) {
            const uint32_t code = p.list[e];
            const uint32_t vi = code >> 1;
            const int mir = int(code & 1u);
            const Item<R> it = p.items[vi];
            int cx, cy;
            item_centre(it, mir, gN, cx, cy);
            t.S = (KMODE == KM_WPROJ) ? p.plane_support[it.plane] : p.support;
            t.K = 2 * t.S + 1;
            t.cpx = it.cpx;
            t.cpy = it.cpy;
            if (mir && gos > 1) {
                t.cpx = gos - t.cpx;
                t.cpy = gos - t.cpy;
            }
            vr = it.vr;
            vim = mir ? -it.vi : it.vi;
            t.wt = it.w;
            rb = cy - t.S;
            cb = cx - t.S;
            // column window of the footprint inside this tile; only footprints
            // crossing the grid edge need the per-tap wrap
            cwrap = cb < 0 || cb + t.K > gN;
            cbase = cb - c0;
            jlo = cwrap ? 0 : max(0, -cbase);
            jhi = cwrap ? t.K : min(t.K, TILE_C - cbase);
            const int krow = ((rb % gN) + gN) % gN, kcol = ((cb % gN) + gN) % gN;
            key = (unsigned long long)krow * (unsigned long long)gN + (unsigned long long)kcol;
            if (KMODE == KM_WPROJ) {
                t.conj_k = (it.flags >> (mir ? 1 : 0)) & 1u;
                t.wconv = p.wk + p.wk_off[it.plane] + uint32_t((t.cpy * p.cs + t.cpx) * t.K * t.K);
            }
            if (KMODE == KM_EXACT) {
                t.fx = p.frac[vi];
                t.fy = p.frac[p.n + vi];
                if (mir) {
                    t.fx *= -1;
                    t.fy *= -1;
                }
                // arma::accu of the column-major outer product (two accumulators)
                double a1 = 0.0, a2 = 0.0;
                int lin = 0;
                for (int c = 0; c < t.K; c++) {
                    const double xc = kernel_value(p.kf, p.trunc, (double(c) - t.S) - t.fx);
                    for (int r = 0; r < t.K; r++, lin++) {
                        const double v = kernel_value(p.kf, p.trunc, (double(r) - t.S) - t.fy) * xc;
                        if (lin & 1)
                            a2 += v;
                        else
                            a1 += v;
                    }
                }
                t.ksum = a1 + a2;
            }
        }
        // rounds: one item per kernel corner per round, so that at every
        // step of the lockstep walk distinct lanes touch distinct cells
        unsigned pending = __ballot_sync(0xffffffffu, active);
        while (pending) {
            const unsigned peers
                = __match_any_sync(0xffffffffu, (active && ((pending >> lane) & 1u)) ? key : ~0ull);
            const bool mine = active && ((pending >> lane) & 1u) && (__ffs(peers & pending) - 1 == lane);
            const unsigned sel = __ballot_sync(0xffffffffu, mine);
            pending &= ~sel;
            int kmax = mine ? t.K : 0;
            for (int o = 16; o > 0; o >>= 1)
                kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
            const bool anywrap = __any_sync(0xffffffffu, mine && cwrap);
            if (KMODE != KM_EXACT && !anywrap && !BEAM) {
                // common case: no footprint of the round crosses the grid's
                // column edge, so each lane's in-tile columns are the window
                // [jl, jh) and tap (i, j) sits at a fixed slot stride; the
                // weight is folded into the visibility once per item
                const int jl = mine ? jlo : 0;
                const int jh = mine ? min(jhi, t.K) : 0;
                const R vrw = vr * t.wt, viw = vim * t.wt;
                for (int i = 0; i < kmax; i++) {
                    const int rm = (mine && i < t.K) ? map_row(rb + i, gN, grows, wrap_neg) : -1;
                    const int rl = rm - r0;
                    const bool rok = rm >= 0 && rl >= 0 && rl < TILE_R;
                    const int jhi_r = rok ? jh : 0;
                    const int slot0 = cbase * TILE_R + rl;
                    for (int j0 = 0; j0 < kmax; j0 += 8) {
                        R kr[8], ki[8];
#pragma unroll
                        for (int jj = 0; jj < 8; jj++) {
                            const int j = j0 + jj;
                            kr[jj] = R(0);
                            ki[jj] = R(0);
                            if (j >= jl && j < jhi_r)
                                tap_value<R, KMODE>(p, tab, t, i, j, kr[jj], ki[jj]);
                        }
#pragma unroll
                        for (int jj = 0; jj < 8; jj++) {
                            const int j = j0 + jj;
                            if (j < kmax) {
                                if (j >= jl && j < jhi_r) {
                                    const R re = vrw * kr[jj] - viw * ki[jj];
                                    const R im = vrw * ki[jj] + viw * kr[jj];
                                    acc_rmw(&acc[slot0 + j * TILE_R], re, im);
                                }
                                __syncwarp();
                            }
                        }
                    }
                }
            } else if (KMODE != KM_EXACT) {
                // tabulated kernels: the lane's kernel row is fetched into
                // registers eight taps at a time, so the loads are in flight
                // together, then accumulated tap by tap in lockstep
                for (int i = 0; i < kmax; i++) {
                    const int rm = (mine && i < t.K) ? map_row(rb + i, gN, grows, wrap_neg) : -1;
                    const int rl = rm - r0;
                    const bool rok = rm >= 0 && rl >= 0 && rl < TILE_R;
                    for (int j0 = 0; j0 < kmax; j0 += 8) {
                        R kr[8], ki[8];
#pragma unroll
                        for (int jj = 0; jj < 8; jj++) {
                            const int j = j0 + jj;
                            kr[jj] = R(0);
                            ki[jj] = R(0);
                            if (rok && j < t.K && j >= jlo && j < jhi) {
                                tap_value<R, KMODE>(p, tab, t, i, j, kr[jj], ki[jj]);
                                kr[jj] = kr[jj] * t.wt;
                                ki[jj] = ki[jj] * t.wt;
                            }
                        }
#pragma unroll
                        for (int jj = 0; jj < 8; jj++) {
                            const int j = j0 + jj;
                            if (j < kmax) {
                                if (rok && j < t.K && j >= jlo && j < jhi) {
                                    const int cl = cwrap ? map_col(cb + j, gN) - c0 : cbase + j;
                                    if (cl >= 0 && cl < TILE_C) {
                                        const R re = vr * kr[jj] - vim * ki[jj];
                                        const R im = vr * ki[jj] + vim * kr[jj];
                                        acc_rmw(&acc[cl * TILE_R + rl], re, im);
                                        if (BEAM)
                                            acc_rmw(&bacc[cl * TILE_R + rl], kr[jj], ki[jj]);
                                    }
                                }
                                __syncwarp();
                            }
                        }
                    }
                }
            } else {
                for (int i = 0; i < kmax; i++) {
                    const int rm = (mine && i < t.K) ? map_row(rb + i, gN, grows, wrap_neg) : -1;
                    const int rl = rm - r0;
                    const bool rok = rm >= 0 && rl >= 0 && rl < TILE_R;
                    for (int j = 0; j < kmax; j++) {
                        if (rok && j < t.K && j >= jlo && j < jhi) {
                            const int cl = cwrap ? map_col(cb + j, gN) - c0 : cbase + j;
                            if (cl >= 0 && cl < TILE_C) {
                                R kr, ki;
                                tap_value<R, KMODE>(p, tab, t, i, j, kr, ki);
                                kr = kr * t.wt;
                                ki = ki * t.wt;
                                const R re = vr * kr - vim * ki;
                                const R im = vr * ki + vim * kr;
                                acc_rmw(&acc[cl * TILE_R + rl], re, im);
                                if (BEAM)
                                    acc_rmw(&bacc[cl * TILE_R + rl], kr, ki);
                            }
                        }
                        __syncwarp();
                    }
                }
            }
        }
    }
    __syncwarp();
    const int nr = min(TILE_R, grows - r0);
    const int nc = min(TILE_C, gN - c0);
    for (int q = lane; q < TILE_R * TILE_C; q += 32) {
        const int rl = q % TILE_R, cl = q / TILE_R;
        if (rl < nr && cl < nc) {
            const size_t g = size_t(c0 + cl) * grows + (r0 + rl);
            cell_store<R, COMP>(p.grid, g, acc[q], p.wide);
            if (BEAM)
                cell_store<R, COMP>(p.beam, g, bacc[q], p.wide);
        }
    }
}

// In-tile part of one footprint axis: taps t in [lo, hi) of raw index
// base + t land on tile positions base + t + shift - origin.  `wrap_pos`:
// raw indices >= N map to raw - N; `wrap_neg`: raw < 0 map to raw + N (else
// they are dropped); only positions < limit exist.  Assumes N is large
// against K + the tile size, so that at most one of the three candidate
// segments meets the tile.
__device__ __forceinline__ void tile_span(int base, int K, int N, int origin, int width, int limit, bool wrap_neg,
    int& lo, int& hi, int& shift)
{
    const int top = min(origin + width, limit); // tile positions [origin, top)
    // non-wrapped raw in [0, N)
    lo = max(max(origin - base, -base), 0);
    hi = min(min(top - base, N - base), K);
    shift = 0;
    if (lo < hi)
        return;
    // raw >= N -> raw - N
    lo = max(max(origin + N - base, N - base), 0);
    hi = min(top + N - base, K);
    shift = -N;
    if (lo < hi)
        return;
    if (wrap_neg) { // raw < 0 -> raw + N
        lo = max(origin - N - base, 0);
        hi = min(min(top - N - base, -base), K);
        shift = N;
        if (lo < hi)
            return;
    }
    lo = hi = 0;
}

// Column-packed tile gridder (tabulated kernels).  One warp per tile.  Each
// list entry (item, mirrored bit) is clipped to the tile: in-tile taps rows
// [ilo, ihi) x columns [jlo, jhi).  A round packs the in-tile columns of
// several entries side by side into the 32 lanes (lane = one column of one
// entry) and walks their rows in lock-step, so lanes are spent on in-tile taps
// only.  Lanes whose cells coincide in one step (two entries of a round
// overlapping) are serialised by __match_any_sync; consecutive steps are
// ordered by __syncwarp.  Requires N >= 2 (Kmax + tile) + 2 (one segment per
// axis and tile); smaller grids use grid_tile.
template <typename R, int COMP, int KMODE, bool BEAM, int TILE_C>
__device__ __forceinline__ void grid_tile_cols(const GridParams<R>& p, int tile, unsigned char* smem_raw)
{
    using A = Acc<R, COMP>;
    using C2 = typename Cplx<R>::T;
    A* acc = reinterpret_cast<A*>(smem_raw);
    A* bacc = acc + (BEAM ? TILE_R * TILE_C : 0);
    R* tab = reinterpret_cast<R*>(acc + (BEAM ? 2 : 1) * TILE_R * TILE_C);
    __shared__ int owner[32];
    const int lane = threadIdx.x;
    const int gN = p.N, grows = p.image_rows, gos = p.os;
    const int tr = tile % p.tiles_r, tc = tile / p.tiles_r;
    const int r0 = tr * TILE_R, c0 = tc * TILE_C;

    for (int t = lane; t < TILE_R * TILE_C; t += 32) {
        acc_zero(&acc[t]);
        if (BEAM)
            acc_zero(&bacc[t]);
    }
    if (KMODE == KM_SEP) {
        const int K = 2 * p.support + 1;
        for (int t = lane; t < p.cs * K; t += 32)
            tab[t] = p.k1d[t];
    }
    __syncwarp();

    const uint32_t beg = p.tile_off[tile], end = p.tile_off[tile + 1];
    for (uint32_t base = beg; base < end; base += 32) {
        // this lane's entry, clipped to the tile
        const uint32_t e = base + lane;
        int K = 1, ilo = 0, nrows = 0, jlo = 0, ncols = 0, rowb = 0, colb = 0;
        uint32_t koff = 0; // W-proj: table offset of the item's K x K kernel; separable: cpy*K << 16 | cpx*K
        R vr = R(0), vi = R(0), wt = R(0);
        int conj = 0;
        if (e < end) {
            const uint32_t code = p.list[e];
            const uint32_t idx = code >> 1;
            const int mir = int(code & 1u);
            const Item<R> it = p.items[idx];
            int cx, cy;
            item_centre(it, mir, gN, cx, cy);
            const int S = (KMODE == KM_WPROJ) ? p.plane_support[it.plane] : p.support;
            K = 2 * S + 1;
            int cpx = it.cpx, cpy = it.cpy;
            if (mir && gos > 1) {
                cpx = gos - cpx;
                cpy = gos - cpy;
            }
            const int rb = cy - S, cb = cx - S;
            int ihi, jhi, rsh, csh;
            tile_span(rb, K, gN, r0, TILE_R, grows, false, ilo, ihi, rsh);
            tile_span(cb, K, gN, c0, TILE_C, gN, true, jlo, jhi, csh);
            nrows = max(ihi - ilo, 0);
            ncols = nrows > 0 ? max(jhi - jlo, 0) : 0;
            rowb = rb + rsh - r0; // local row of tap i: rowb + i
            colb = cb + csh - c0; // local column of tap j: colb + j
            vr = it.vr;
            vi = mir ? -it.vi : it.vi;
            wt = it.w;
            if (KMODE == KM_WPROJ) {
                conj = (it.flags >> (mir ? 1 : 0)) & 1u;
                koff = p.wk_off[it.plane] + uint32_t((cpy * p.cs + cpx) * K * K);
            } else {
                koff = (uint32_t(cpy * K) << 16) | uint32_t(cpx * K);
            }
        }
        const R vrw = vr * wt, viw = vi * wt;
        bool pending = ncols > 0;
        while (__any_sync(0xffffffffu, pending)) {
            // pack a prefix of the pending entries into the lanes
            const int x = pending ? ncols : 0;
            int incl = x;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o)
                    incl += y;
            }
            const bool take = pending && incl <= 32;
            const int off = incl - x;
            if (take)
                for (int t = 0; t < ncols; t++)
                    owner[off + t] = lane;
            int total = take ? incl : 0, steps = take ? nrows : 0;
            for (int o = 16; o > 0; o >>= 1) {
                total = max(total, __shfl_xor_sync(0xffffffffu, total, o));
                steps = max(steps, __shfl_xor_sync(0xffffffffu, steps, o));
            }
            __syncwarp();
            const int own = lane < total ? owner[lane] : lane;
            __syncwarp();
            const bool mine = lane < total;
            // the owner entry's parameters
            const int o_ilo = __shfl_sync(0xffffffffu, ilo, own);
            const int o_nrows = __shfl_sync(0xffffffffu, nrows, own);
            const int o_jlo = __shfl_sync(0xffffffffu, jlo, own);
            const int o_off = __shfl_sync(0xffffffffu, off, own);
            const int o_rowb = __shfl_sync(0xffffffffu, rowb, own);
            const int o_colb = __shfl_sync(0xffffffffu, colb, own);
            const int o_K = __shfl_sync(0xffffffffu, K, own);
            const uint32_t o_koff = __shfl_sync(0xffffffffu, koff, own);
            const R o_vr = __shfl_sync(0xffffffffu, vrw, own);
            const R o_vi = __shfl_sync(0xffffffffu, viw, own);
            const R o_wt = BEAM ? __shfl_sync(0xffffffffu, wt, own) : R(0);
            const int o_conj = __shfl_sync(0xffffffffu, conj, own);
            const int j = o_jlo + (lane - o_off);
            const int col = o_colb + j;
            for (int st = 0; st < steps; st++) {
                const bool act = mine && st < o_nrows;
                const int i = o_ilo + st;
                R kr = R(0), ki = R(0);
                if (act) {
                    if (KMODE == KM_WPROJ) {
                        const C2 v = p.wk[o_koff + uint32_t(i * o_K + j)];
                        kr = v.x;
                        ki = o_conj ? -v.y : v.y;
                    } else {
                        kr = tab[(o_koff >> 16) + uint32_t(i)] * tab[(o_koff & 0xffffu) + uint32_t(j)];
                    }
                }
                const int slot = col * TILE_R + (o_rowb + i);
                bool todo = act;
                while (__any_sync(0xffffffffu, todo)) {
                    const unsigned peers = __match_any_sync(0xffffffffu, todo ? slot : -1 - lane);
                    const bool lead = todo && (__ffs(peers) - 1 == lane);
                    if (lead) {
                        const R re = o_vr * kr - o_vi * ki;
                        const R im = o_vr * ki + o_vi * kr;
                        acc_rmw(&acc[slot], re, im);
                        if (BEAM)
                            acc_rmw(&bacc[slot], kr * o_wt, ki * o_wt);
                    }
                    todo = todo && !lead;
                    __syncwarp();
                }
            }
            pending = pending && !take;
        }
    }
    __syncwarp();
    const int nr = min(TILE_R, grows - r0);
    const int nc = min(TILE_C, gN - c0);
    for (int q = lane; q < TILE_R * TILE_C; q += 32) {
        const int rl = q % TILE_R, cl = q / TILE_R;
        if (rl < nr && cl < nc) {
            const size_t g = size_t(c0 + cl) * grows + (r0 + rl);
            cell_store<R, COMP>(p.grid, g, acc[q], p.wide);
            if (BEAM)
                cell_store<R, COMP>(p.beam, g, bacc[q], p.wide);
        }
    }
}

// One CTA (one warp) per tile of one snapshot.
// Residency target: the shared-memory tile allows ~28 CTAs per SM at 16
// columns (8 KB FP32/FP32C cell tile) and ~14 at 32; registers are capped to match.
// Lane-per-tap tile gridder (tabulated kernels).  One warp per tile; the
// 32 list entries of a batch are clipped to the tile by their own lanes
// (window rows [ilo, ihi) x columns [jlo, jhi)), then taken one at a time:
// the entry's parameters are broadcast and its in-tile taps are spread over
// the lanes, 32 per pass (lane = tap, column-major in the window, so that
// consecutive lanes touch consecutive accumulator cells).  All taps of one
// pass hit distinct cells, so there are no conflicts; consecutive passes are
// ordered by __syncwarp.  Every lane does useful work on windows of 32 taps
// or more; small kernels (K = 5 or 7 at one tile per footprint) fill most of
// a pass.  Requires N >= 2 (Kmax + tile) + 2, as grid_tile_cols.
template <typename R, int COMP, int KMODE, bool BEAM, int TILE_C>
__device__ __forceinline__ void grid_tile_taps(const GridParams<R>& p, int tile, unsigned char* smem_raw)
{
    using A = Acc<R, COMP>;
    using C2 = typename Cplx<R>::T;
    A* acc = reinterpret_cast<A*>(smem_raw);
    A* bacc = acc + (BEAM ? TILE_R * TILE_C : 0);
    R* tab = reinterpret_cast<R*>(acc + (BEAM ? 2 : 1) * TILE_R * TILE_C);
    const int lane = threadIdx.x & 31;
    const int gN = p.N, grows = p.image_rows, gos = p.os;
    const int tr = tile % p.tiles_r, tc = tile / p.tiles_r;
    const int r0 = tr * TILE_R, c0 = tc * TILE_C;

    for (int t = lane; t < TILE_R * TILE_C; t += 32) {
        acc_zero(&acc[t]);
        if (BEAM)
            acc_zero(&bacc[t]);
    }
    if (KMODE == KM_SEP) {
        const int K = 2 * p.support + 1;
        for (int t = lane; t < p.cs * K; t += 32)
            tab[t] = p.k1d[t];
    }
    __syncwarp();

    const uint32_t beg = p.tile_off[tile], end = p.tile_off[tile + 1];
    for (uint32_t base = beg; base < end; base += 32) {
        // this lane's entry, clipped to the tile
        const uint32_t e = base + lane;
        int K = 1, ilo = 0, nrows = 0, jlo = 0, ncols = 0, rowb = 0, colb = 0;
        uint32_t koff = 0; // W-proj: table offset of the item's K x K kernel; separable: cpy*K << 16 | cpx*K
        R vr = R(0), vi = R(0), wt = R(0);
        int conj = 0;
        if (e < end) {
            const uint32_t code = p.list[e];
            const uint32_t idx = code >> 1;
            const int mir = int(code & 1u);
            const Item<R> it = p.items[idx];
            int cx, cy;
            item_centre(it, mir, gN, cx, cy);
            const int S = (KMODE == KM_WPROJ) ? p.plane_support[it.plane] : p.support;
            K = 2 * S + 1;
            int cpx = it.cpx, cpy = it.cpy;
            if (mir && gos > 1) {
                cpx = gos - cpx;
                cpy = gos - cpy;
            }
            const int rb = cy - S, cb = cx - S;
            int ihi, jhi, rsh, csh;
            tile_span(rb, K, gN, r0, TILE_R, grows, false, ilo, ihi, rsh);
            tile_span(cb, K, gN, c0, TILE_C, gN, true, jlo, jhi, csh);
            nrows = max(ihi - ilo, 0);
            ncols = nrows > 0 ? max(jhi - jlo, 0) : 0;
            if (ncols == 0)
                nrows = 0;
            rowb = rb + rsh - r0; // local row of tap i: rowb + i
            colb = cb + csh - c0; // local column of tap j: colb + j
            vr = it.vr;
            vi = mir ? -it.vi : it.vi;
            wt = it.w;
            if (KMODE == KM_WPROJ) {
                conj = (it.flags >> (mir ? 1 : 0)) & 1u;
                koff = p.wk_off[it.plane] + uint32_t((cpy * p.cs + cpx) * K * K);
            } else {
                koff = (uint32_t(cpy * K) << 16) | uint32_t(cpx * K);
            }
        }
        const R vrw = vr * wt, viw = vi * wt;
        const int nt = nrows * ncols;
        const int np = (nt + 31) >> 5;
        // passes of the batch: unit u belongs to the last lane whose start <= u
        int incl = np;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        const int start = incl - np;
        const int units = __shfl_sync(0xffffffffu, incl, 31);
        // packed per-entry words for the broadcasts
        const int geo = (ilo & 0xff) | ((jlo & 0xff) << 8) | ((nrows & 0xff) << 16) | ((conj & 1) << 24);
        const int loc = (rowb & 0xffff) | int(unsigned(colb) << 16);
        const int kn = (K & 0xffff) | (nt << 16);
        const float rcp = nrows > 0 ? 1.0f / float(nrows) : 0.0f;
        for (int u = 0; u < units; u++) {
            const unsigned le = __ballot_sync(0xffffffffu, np > 0 && start <= u);
            const int own = 31 - __clz(le);
            const int pass = u - __shfl_sync(0xffffffffu, start, own);
            const int o_geo = __shfl_sync(0xffffffffu, geo, own);
            const int o_loc = __shfl_sync(0xffffffffu, loc, own);
            const int o_kn = __shfl_sync(0xffffffffu, kn, own);
            const uint32_t o_koff = __shfl_sync(0xffffffffu, koff, own);
            const float o_rcp = __shfl_sync(0xffffffffu, rcp, own);
            const R o_vr = __shfl_sync(0xffffffffu, vrw, own);
            const R o_vi = __shfl_sync(0xffffffffu, viw, own);
            const R o_wt = BEAM ? __shfl_sync(0xffffffffu, wt, own) : R(0);
            const int o_nt = o_kn >> 16, o_K = o_kn & 0xffff;
            const int t = pass * 32 + lane;
            if (t < o_nt) {
                // window column-major: consecutive lanes take consecutive rows,
                // i.e. consecutive accumulator cells
                const int o_nrows = (o_geo >> 16) & 0xff;
                const int dj = int((float(t) + 0.5f) * o_rcp);
                const int di = t - dj * o_nrows;
                const int i = (o_geo & 0xff) + di, j = ((o_geo >> 8) & 0xff) + dj;
                R kr, ki;
                if (KMODE == KM_WPROJ) {
                    const C2 v = p.wk[o_koff + uint32_t(i * o_K + j)];
                    kr = v.x;
                    ki = ((o_geo >> 24) & 1) ? -v.y : v.y;
                } else {
                    kr = tab[(o_koff >> 16) + uint32_t(i)] * tab[(o_koff & 0xffffu) + uint32_t(j)];
                    ki = R(0);
                }
                const int row = int(short(o_loc & 0xffff)) + i, col = (o_loc >> 16) + j;
                const int slot = col * TILE_R + row;
                const R re = o_vr * kr - o_vi * ki;
                const R im = o_vr * ki + o_vi * kr;
                acc_rmw(&acc[slot], re, im);
                if (BEAM)
                    acc_rmw(&bacc[slot], kr * o_wt, ki * o_wt);
            }
            __syncwarp();
        }
    }
    __syncwarp();
    const int nr = min(TILE_R, grows - r0);
    const int nc = min(TILE_C, gN - c0);
    for (int q = lane; q < TILE_R * TILE_C; q += 32) {
        const int rl = q % TILE_R, cl = q / TILE_R;
        if (rl < nr && cl < nc) {
            const size_t g = size_t(c0 + cl) * grows + (r0 + rl);
            cell_store<R, COMP>(p.grid, g, acc[q], p.wide);
            if (BEAM)
                cell_store<R, COMP>(p.beam, g, bacc[q], p.wide);
        }
    }
}

// ---------------------------------------------------------------- staged gridder

// Record fill: like k_fill_tiles, but each (entry, tile) pair is written as a
// decoded TapRec at its slot of the tile's range (tile order), the footprint
// already clipped to the tile (tile_span, as grid_tile_taps clips it).  Slots
// beyond `cap` are not written and set bit 8 of *err (the caller grows the
// buffer to the counted total and grids again).
template <typename R>
struct RecFill {
    TapRec<R>* rec;
    uint64_t cap;
    const uint32_t* wk_off; // W-projection: table offset per plane (x time step)
    int cs, os;
};

template <typename R, int KMODE>
__global__ void k_fill_recs(BinParams p, Item<R>* items, const uint32_t* order, const int64_t* first, int P,
    RecFill<R> q)
{
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= p.n)
        return;
    const Item<R> it = items[k];
    if (!it.good)
        return;
    int S = p.support, plane = 0;
    if (p.plane16) {
        plane = p.plane16[k];
        S = p.plane_support[plane];
        items[k].plane = uint16_t(plane);
    } else if (order) {
        plane = plane_of(first, P, k);
        if (p.ts_of)
            plane = plane * p.ntimesteps + p.ts_of[order[k]];
        S = p.plane_support[plane];
        items[k].plane = uint16_t(plane);
    }
    const int K = 2 * S + 1;
    const bool ranked = p.ranks && *p.rank_overflow == 0u;
    for (int mir = 0; mir < int(it.good); mir++) {
        int cx, cy;
        item_centre(it, mir, p.N, cx, cy);
        int cpx = it.cpx, cpy = it.cpy;
        if (mir && q.os > 1) {
            cpx = q.os - cpx;
            cpy = q.os - cpy;
        }
        TapRec<R> r;
        r.vr = it.vr * it.w;
        r.vi = (mir ? -it.vi : it.vi) * it.w;
        const int conj = KMODE == KM_WPROJ ? int((it.flags >> (mir ? 1 : 0)) & 1u) : 0;
        const uint32_t kbase = KMODE == KM_WPROJ ? q.wk_off[plane] + uint32_t((cpy * q.cs + cpx) * K * K) : 0u;
        const int rb = cy - S, cb = cx - S;
        int qn = 0;
        for_item_tiles(it, mir, S, p, [&](uint32_t t) {
            const uint32_t slot = ranked ? p.ranks[size_t(qn * 2 + mir) * size_t(p.n) + size_t(k)]
                                         : atomicAdd(&p.tile_cursor[t], 1u);
            qn++;
            const int r0 = int(t % uint32_t(p.tiles_r)) * TILE_R, c0 = int(t / uint32_t(p.tiles_r)) * p.tile_c;
            int ilo, ihi, rsh, jlo, jhi, csh;
            tile_span(rb, K, p.N, r0, TILE_R, p.image_rows, false, ilo, ihi, rsh);
            tile_span(cb, K, p.N, c0, p.tile_c, p.N, true, jlo, jhi, csh);
            int nrows = max(ihi - ilo, 0), ncols = max(jhi - jlo, 0);
            if (nrows == 0 || ncols == 0)
                nrows = ncols = 0;
            const int row0 = nrows ? rb + rsh - r0 + ilo : 0;
            const int col0 = ncols ? cb + csh - c0 + jlo : 0;
            r.koff = KMODE == KM_WPROJ ? kbase + uint32_t(ilo * K + jlo)
                                       : (uint32_t(cpy * K + ilo) << 16) | uint32_t(cpx * K + jlo);
            r.geom = rec_geom(row0, col0, nrows, ncols, conj, K);
            const uint64_t pos = uint64_t(p.tile_off[t]) + slot;
            if (pos < q.cap)
                q.rec[pos] = r;
            else
                atomicOr(p.err, 8u);
        });
    }
}

// Bulk (TMA) copies into shared memory completing on an mbarrier, and a
// bounded wait for a barrier phase.
constexpr int kRecChunk = 64;              // records per staged chunk (two chunks in flight per warp)
constexpr uint32_t kWaitLimit = 1u << 22; // try_wait rounds before a wait gives up

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(1u) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// one arrival that expects `bytes`, then the copy that delivers them
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < kWaitLimit; it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

// ceil(65536 / n), n = 1..32: (t * m) >> 16 == t / n for t < 1024
__constant__ uint32_t c_div_magic[33] = { 0, 65536, 32768, 21846, 16384, 13108, 10923, 9363, 8192, 7282, 6554, 5958,
    5462, 5042, 4682, 4370, 4096, 3856, 3641, 3450, 3277, 3121, 2979, 2850, 2731, 2622, 2521, 2428, 2341, 2260, 2185,
    2115, 2048 };

// Shared memory of one warp of the staged gridder: accumulators, two record
// buffers, two barriers and the separable kernel table.
template <typename R, int COMP, int TILE_C>
__host__ __device__ constexpr size_t rec_warp_bytes(int sep_table_len)
{
    return ((sizeof(Acc<R, COMP>) * TILE_R * TILE_C + 2 * kRecChunk * sizeof(TapRec<R>) + 16
                + sizeof(R) * size_t(sep_table_len))
               + 15)
        / 16 * 16;
}

// Staged tile gridder: one warp per tile.  The tile's records (k_fill_recs)
// arrive in chunks of kRecChunk by bulk copies into two shared-memory
// buffers (the next chunk is in flight while one is processed); the warp
// takes the entries one at a time, each lane one tap of the entry's clipped
// window (column-major, so consecutive lanes update consecutive cells: the
// taps of one entry are distinct cells, entries are ordered by __syncwarp),
// the record read from shared memory by all lanes at once.  Accumulation,
// zeroing and the single coalesced store are those of grid_tile_taps.  A
// barrier wait that gives up (never expected) sets bit 16 of *err, waits for
// the copies still in flight and leaves the tile unwritten.
template <typename R, int COMP, int KMODE, int TILE_C>
__device__ __forceinline__ bool grid_tile_recs(const GridParams<R>& p, int tile, unsigned char* smem_raw)
{
    unsigned int* err = p.err;
    using A = Acc<R, COMP>;
    using C2 = typename Cplx<R>::T;
    A* acc = reinterpret_cast<A*>(smem_raw);
    TapRec<R>* rbuf = reinterpret_cast<TapRec<R>*>(acc + TILE_R * TILE_C);
    uint64_t* bar = reinterpret_cast<uint64_t*>(rbuf + 2 * kRecChunk);
    R* tab = reinterpret_cast<R*>(bar + 2);
    const int lane = threadIdx.x & 31;
    const int gN = p.N, grows = p.image_rows;
    const int tr = tile % p.tiles_r, tc = tile / p.tiles_r;
    const int r0 = tr * TILE_R, c0 = tc * TILE_C;
    const uint32_t beg = p.tile_off[tile];
    uint32_t cnt = p.tile_off[tile + 1] - beg;
    if (uint64_t(beg) + cnt > p.rec_cap) { // the fill overflowed (bit 8 is set): copy nothing
        cnt = 0;
        if (lane == 0)
            atomicOr(err, 8u);
    }
    const int nch = int((cnt + kRecChunk - 1) / kRecChunk);
    auto issue = [&](int c) {
        const uint32_t n = min(uint32_t(kRecChunk), cnt - uint32_t(c) * kRecChunk);
        bulk_copy_g2s(rbuf + (c & 1) * kRecChunk, p.recs + beg + uint32_t(c) * kRecChunk,
            n * uint32_t(sizeof(TapRec<R>)), &bar[c & 1]);
    };
    if (lane == 0) {
        mbar_init(&bar[0]);
        mbar_init(&bar[1]);
        mbar_init_fence();
        if (nch > 0)
            issue(0);
        if (nch > 1)
            issue(1);
    }
    for (int t = lane; t < TILE_R * TILE_C; t += 32)
        acc_zero(&acc[t]);
    if (KMODE == KM_SEP) {
        const int K = 2 * p.support + 1;
        for (int t = lane; t < p.cs * K; t += 32)
            tab[t] = p.k1d[t];
    }
    __syncwarp();
    for (int c = 0; c < nch; c++) {
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&bar[c & 1], uint32_t(c >> 1) & 1u));
        if (!ok) {
            if (lane == 0) {
                // record the failure, then wait (bounded again) for this
                // chunk's copy and the other buffer's before leaving
                atomicOr(err, 16u);
                mbar_wait(&bar[c & 1], uint32_t(c >> 1) & 1u);
                if (c + 1 < nch)
                    mbar_wait(&bar[(c + 1) & 1], uint32_t((c + 1) >> 1) & 1u);
            }
            __syncwarp();
            return false;
        }
        const TapRec<R>* rb = rbuf + (c & 1) * kRecChunk;
        const int ne = min(kRecChunk, int(cnt) - c * kRecChunk);
        // an entry decoded once: window shape, divisor magic, first cell,
        // kernel offsets and the weighted visibility (pvr, pvi: its parts
        // negated when the W-kernel is conjugated, so that the product
        // needs no per-tap sign)
        struct Ent {
            int nrows, nt, sbase, K;
            uint32_t m, koff, ky, kx;
            R vr, vi, pvr, pvi;
        };
        auto decode = [&](const TapRec<R>& r) {
            Ent x;
            const uint32_t g = r.geom;
            x.nrows = int((g >> 10) & 63u);
            x.nt = x.nrows * int((g >> 16) & 63u);
            x.m = c_div_magic[x.nrows];
            x.sbase = int((g >> 5) & 31u) * TILE_R + int(g & 31u);
            x.K = int(g >> 23);
            const bool conj = (g >> 22) & 1u;
            x.koff = r.koff;
            x.ky = r.koff >> 16;
            x.kx = r.koff & 0xffffu;
            x.vr = r.vr;
            x.vi = r.vi;
            x.pvr = conj ? -r.vr : r.vr;
            x.pvi = conj ? -r.vi : r.vi;
            return x;
        };
        // tap t of an entry: its accumulator cell and weighted value
        auto tap = [&](const Ent& x, int t, int& cell, R& re, R& im) {
            const int dj = int((uint32_t(t) * x.m) >> 16);
            const int di = t - dj * x.nrows;
            if (KMODE == KM_WPROJ) {
                // (vr + i vi)(kr + i ki), ki = -v.y for a conjugated kernel
                const C2 v = __ldg(&p.wk[x.koff + uint32_t(di * x.K + dj)]);
                re = x.vr * R(v.x) - x.pvi * R(v.y);
                im = x.pvr * R(v.y) + x.vi * R(v.x);
            } else {
                const R kr = tab[x.ky + uint32_t(di)] * tab[x.kx + uint32_t(dj)];
                re = x.vr * kr;
                im = x.vi * kr;
            }
            cell = x.sbase + dj * TILE_R + di;
        };
        // two single-pass entries at a time where possible: both kernel
        // loads in flight before either entry's cells are updated
        for (int e = 0; e < ne;) {
            const Ent ea = decode(rb[e]);
            if (ea.nt <= 32 && e + 1 < ne) {
                const Ent eb = decode(rb[e + 1]);
                if (eb.nt <= 32) {
                    int ca = 0, cb = 0;
                    R xa = R(0), ya = R(0), xb = R(0), yb = R(0);
                    const bool ia = lane < ea.nt, ib = lane < eb.nt;
                    if (ia)
                        tap(ea, lane, ca, xa, ya);
                    if (ib)
                        tap(eb, lane, cb, xb, yb);
                    if (ia)
                        acc_rmw(&acc[ca], xa, ya);
                    __syncwarp();
                    if (ib)
                        acc_rmw(&acc[cb], xb, yb);
                    __syncwarp();
                    e += 2;
                    continue;
                }
            }
            // an entry's taps are distinct cells: up to four passes' kernel
            // loads are issued before their updates, with no ordering
            // between the passes
            for (int t0 = lane; t0 < ea.nt; t0 += 128) {
                int cell[4];
                R xr[4], yi[4];
                bool in[4];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    in[q] = t0 + q * 32 < ea.nt;
                    if (in[q])
                        tap(ea, t0 + q * 32, cell[q], xr[q], yi[q]);
                }
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (in[q])
                        acc_rmw(&acc[cell[q]], xr[q], yi[q]);
            }
            __syncwarp();
            e++;
        }
        if (lane == 0 && c + 2 < nch) {
            // the buffer's records were read by every lane (ordered by the
            // __syncwarp above) before the async proxy overwrites it
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(c + 2);
        }
        __syncwarp();
    }
    const int nr = min(TILE_R, grows - r0);
    const int nc = min(TILE_C, gN - c0);
    for (int q = lane; q < TILE_R * TILE_C; q += 32) {
        const int rl = q % TILE_R, cl = q / TILE_R;
        if (rl < nr && cl < nc) {
            cell_store<R, COMP>(p.grid, size_t(c0 + cl) * grows + (r0 + rl), acc[q], p.wide);
        }
    }
    // every copy has completed: the barriers can be initialised again for
    // the warp's next tile (persistent batch gridder)
    if (lane == 0) {
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar[0])) : "memory");
        asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&bar[1])) : "memory");
    }
    __syncwarp();
    return true;
}

// Staged gridder with WPB warps per block, each on its own tile (tile
// blockIdx.x * WPB + warp; its shared memory at warp * warp_bytes).
template <typename R, int COMP, int KMODE, int TILE_C, int WPB>
__global__ void __launch_bounds__(32 * WPB) k_grid_tiles_recs(GridParams<R> p, int ntiles, int warp_bytes)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5;
    const int tile = int(blockIdx.x) * WPB + warp;
    if (tile < ntiles)
        grid_tile_recs<R, COMP, KMODE, TILE_C>(p, tile, smem_raw + size_t(warp) * size_t(warp_bytes));
}

// Lane-per-tap gridder with WPB warps per block, each on its own tile (tile
// blockIdx.x * WPB + warp, its accumulators at warp * tile_bytes): narrow
// tiles keep the shared memory per warp small, and several warps per block
// raise the resident warps past the per-SM block limit.
template <typename R, int COMP, int KMODE, bool BEAM, int TILE_C, int WPB>
__global__ void __launch_bounds__(32 * WPB, 44 / WPB) k_grid_tiles_mw(GridParams<R> p, int ntiles, int tile_bytes)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5;
    const int tile = int(blockIdx.x) * WPB + warp;
    if (tile < ntiles)
        grid_tile_taps<R, COMP, KMODE, BEAM, TILE_C>(p, tile, smem_raw + size_t(warp) * size_t(tile_bytes));
}

// FORM: 0 lanes-per-item (grid_tile), 1 column-packed (grid_tile_cols),
// 2 lane-per-tap (grid_tile_taps); the exact gridder always uses grid_tile.
template <typename R, int COMP, int KMODE, bool BEAM, int TILE_C, int FORM = 0>
__global__ void __launch_bounds__(32, TILE_C == 16 ? (sizeof(R) == 8 ? 24 : 28) : 14) k_grid_tiles(GridParams<R> p)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    if constexpr (FORM == 1 && KMODE != KM_EXACT)
        grid_tile_cols<R, COMP, KMODE, BEAM, TILE_C>(p, int(blockIdx.x), smem_raw);
    else if constexpr (FORM == 2 && KMODE != KM_EXACT)
        grid_tile_taps<R, COMP, KMODE, BEAM, TILE_C>(p, int(blockIdx.x), smem_raw);
    else
        grid_tile<R, COMP, KMODE, BEAM, TILE_C>(p, int(blockIdx.x), smem_raw);
}

// Parameters of one persistent gridder launch: up to kBatchGrid snapshots,
// passed by value (kernel parameter space, read through the constant cache
// with a warp-uniform index).
constexpr int kBatchGrid = 64;
template <typename R>
struct BatchGridParams {
    GridParams<R> ps[kBatchGrid];
    uint32_t tile_base[kBatchGrid + 1];
    int nsnap;
    uint32_t* counter;
};

// Persistent gridder over the tiles of many snapshots: a (snapshot, tile)
// work queue.  Work item w is tile w - tile_base[s] of the snapshot s with
// tile_base[s] <= w < tile_base[s + 1]; warps take items from one atomic
// counter (zeroed before the launch) until the queue is empty.
// PERSIST = false: one CTA per work item (w = blockIdx.x), the hardware
// block scheduler being the queue; the autotuner picks the faster form.
template <typename R, int COMP, int KMODE, bool BEAM, int TILE_C, bool PERSIST, int FORM = 0>
__global__ void __launch_bounds__(32, TILE_C == 16 ? (sizeof(R) == 8 ? 24 : 28) : 14) k_grid_batch(const __grid_constant__ BatchGridParams<R> P)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t total = P.tile_base[P.nsnap];
    for (int once = 0;; once++) {
        uint32_t w = 0;
        if (PERSIST) {
            if (threadIdx.x == 0)
                w = atomicAdd(P.counter, 1u);
            w = __shfl_sync(0xffffffffu, w, 0);
        } else {
            if (once)
                break;
            w = blockIdx.x;
        }
        if (w >= total)
            break;
        int lo = 0, hi = P.nsnap - 1;
        while (lo < hi) { // last snapshot whose first tile <= w
            const int mid = (lo + hi + 1) / 2;
            if (P.tile_base[mid] <= w)
                lo = mid;
            else
                hi = mid - 1;
        }
        __syncwarp();
        if constexpr (FORM == 3 && KMODE != KM_EXACT && !BEAM) {
            if (!grid_tile_recs<R, COMP, KMODE, TILE_C>(P.ps[lo], int(w - P.tile_base[lo]), smem_raw))
                break; // a staged copy's wait gave up (flagged): this warp stops
        } else if constexpr (FORM == 2 && KMODE != KM_EXACT)
            grid_tile_taps<R, COMP, KMODE, BEAM, TILE_C>(P.ps[lo], int(w - P.tile_base[lo]), smem_raw);
        else
            grid_tile<R, COMP, KMODE, BEAM, TILE_C>(P.ps[lo], int(w - P.tile_base[lo]), smem_raw);
        __syncwarp();
    }
}

// ---------------------------------------------------------------- kernel tables

// make_1D_kernel for every oversampled offset (populate_kernel_cache,
// gridder.h:73-105): out[cs][K], normalised by accu (two accumulators).
__global__ void k_kernel_table(int kf, double trunc, int support, int os, double* out)
{
    const int half = os / 2;
    const int cs = half * 2 + 1;
    const int K = 2 * support + 1;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cs)
        return;
    const double offset = (double(c) - half) / os;
    double a1 = 0.0, a2 = 0.0;
    for (int i = 0; i < K; i++) {
        double d = (double(i) - support) / 1;
        double v = kernel_value(kf, trunc, d - offset);
        out[c * K + i] = v;
        if (i & 1)
            a2 += v;
        else
            a1 += v;
    }
    const double s = a1 + a2;
    for (int i = 0; i < K; i++)
        out[c * K + i] = out[c * K + i] / s;
}

__global__ void k_d2f(const double* in, float* out, int64_t n)
{
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = float(in[i]);
}

// ImgDomKernel (conv_func.h:351-412).  Analytic: gcf((i - c)/c).  Otherwise
// the real part of the R2HC DFT of the normalised, wrapped 1-D kernel,
// mirrored about the centre.  The kernel is exactly zero beyond `trunc`, so
// the DFT is a short cosine sum, evaluated with exact argument reduction.
__global__ void k_imgdom_kernel(int kf, double trunc, int n, int analytic, double ksum_inv, int dmax, double* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int centre = n / 2;
    if (analytic) {
        out[i] = gcf_value(kf, (double(i) - centre) / centre);
        return;
    }
    // aa[n/2 + m] = r_m (m < n/2), aa[n/2 - m] = r_m (1 <= m <= n/2)
    int m = i >= centre ? i - centre : centre - i;
    double r = 0.0;
    // arr[j] = k1(j) (j < n/2), k1(j - n) (j >= n/2); r_m = sum_j arr[j] cos(2 pi j m / n)
    for (int d = -dmax; d <= dmax; d++) {
        if (d < -centre || d >= n - centre)
            continue;
        double kv = kernel_value(kf, trunc, double(d));
        if (kv == 0.0)
            continue;
        kv = kv * ksum_inv;
        long long jm = (long long)(d < 0 ? d + n : d) * m % n;
        r += kv * cospi(2.0 * double(jm) / double(n));
    }
    out[i] = r;
}

// ---------------------------------------------------------------- normalise

// normalise_image_beam_result_1D, non-FFTSHIFT branch (imager.h:97-150):
// crop the padded image keeping the unshifted quadrant layout, multiply by
// 1/sum and divide by gcf[ii]*gcf[jj].  blockIdx.y = output column; the
// factor 1/sum is read from the device (0 when the sampling total is 0).
template <typename RI, typename RO>
__global__ void __launch_bounds__(256) k_normalise(const RI* __restrict__ img, int padded, int image_size,
    const double* total, const double* __restrict__ ginv, int corr, RO* __restrict__ out)
{
    const int j = blockIdx.y;
    const double tot = total[0];
    const double nf = tot > 0.0 ? 1.0 / tot : 0.0;
    const int hp = padded / 2, hs = image_size / 2;
    const int oj = j < hs ? j : padded + j - image_size;
    const int jj = j < hs ? j + hp : hp + j - image_size;
    // value * (1/sum) / (gcf[ii] * gcf[jj]) as value * (nf * 1/gcf[jj]) * 1/gcf[ii]
    const double fj = corr ? nf * ginv[jj] : nf;
    const RI* src = img + size_t(oj) * padded;
    RO* dst = out + size_t(j) * image_size;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < image_size; i += gridDim.x * blockDim.x) {
        const int oi = i < hs ? i : padded - hs + (i - hs);
        const int ii = i < hs ? hp + i : hp - hs + (i - hs);
        const double v = double(src[oi]) * fj;
        dst[i] = RO(corr ? v * ginv[ii] : v);
    }
}

// Same pass, four rows per thread with 16-byte loads and stores, for
// image_size % 8 == 0 and padded % 4 == 0 (each group of four rows then lies
// inside one crop segment and is 16-byte aligned).  blockIdx.y = a group of
// kNormCols output columns: a thread keeps its rows' 1/gcf for all of them
// and has their loads in flight together (one short block per column spent
// more time in block scheduling than in the copy).
constexpr int kNormCols = 8;
template <typename RI, typename RO>
__global__ void __launch_bounds__(256) k_normalise4(const RI* __restrict__ img, int padded, int image_size,
    const double* total, const double* __restrict__ ginv, int corr, RO* __restrict__ out)
{
    const double tot = total[0];
    const double nf = tot > 0.0 ? 1.0 / tot : 0.0;
    const int hp = padded / 2, hs = image_size / 2;
    const int groups = image_size / 4;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += gridDim.x * blockDim.x) {
        const int i = g * 4;
        const int oi = i < hs ? i : padded - hs + (i - hs);
        const int ii = i < hs ? hp + i : hp - hs + (i - hs);
        double gi[4];
#pragma unroll
        for (int k = 0; k < 4; k++)
            gi[k] = corr ? ginv[ii + k] : 1.0;
        RI x[kNormCols][4];
#pragma unroll
        for (int c = 0; c < kNormCols; c++) {
            const int j = blockIdx.y * kNormCols + c;
            if (j >= image_size)
                break;
            const int oj = j < hs ? j : padded + j - image_size;
            const RI* src = img + size_t(oj) * padded + oi;
            if constexpr (sizeof(RI) == 4) {
                const float4 q = *reinterpret_cast<const float4*>(src);
                x[c][0] = q.x;
                x[c][1] = q.y;
                x[c][2] = q.z;
                x[c][3] = q.w;
            } else {
                const double2 a = *reinterpret_cast<const double2*>(src);
                const double2 b = *reinterpret_cast<const double2*>(src + 2);
                x[c][0] = a.x;
                x[c][1] = a.y;
                x[c][2] = b.x;
                x[c][3] = b.y;
            }
        }
#pragma unroll
        for (int c = 0; c < kNormCols; c++) {
            const int j = blockIdx.y * kNormCols + c;
            if (j >= image_size)
                break;
            const int jj = j < hs ? j + hp : hp + j - image_size;
            const double fj = corr ? nf * ginv[jj] : nf;
            double v[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                v[k] = double(x[c][k]) * fj;
                if (corr)
                    v[k] *= gi[k];
            }
            RO* dst = out + size_t(j) * image_size + i;
            if constexpr (sizeof(RO) == 4) {
                *reinterpret_cast<float4*>(dst) = make_float4(float(v[0]), float(v[1]), float(v[2]), float(v[3]));
            } else {
                *reinterpret_cast<double2*>(dst) = make_double2(v[0], v[1]);
                *reinterpret_cast<double2*>(dst + 2) = make_double2(v[2], v[3]);
            }
        }
    }
}

__global__ void k_reciprocal(const double* in, double* out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = 1.0 / in[i];
}

// ---------------------------------------------------------------- W-projection

// Plane boundaries and plane w (average_w_planes, gridder.cpp:68-146) from the
// |w|-sorted order: cgood[k] = number of good visibilities among sorted[0..k).
__global__ void k_wplanes(const uint32_t* cgood, const double* absw_sorted, int64_t n, int P, int median,
    int64_t* first, int64_t* last)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    const uint64_t G = cgood[n];
    uint64_t begin = 0;
    if (G == uint64_t(n)) {
        // every visibility is in bounds: sorted position == good count
        for (int idx = 0; idx < P; idx++) {
            const uint64_t plane_size = uint64_t(ceil(double(G - begin) / (P - idx)));
            const uint64_t lo = min(uint64_t(n), begin + plane_size);
            first[idx] = int64_t(begin);
            last[idx] = int64_t(lo);
            begin = lo;
        }
        return;
    }
    for (int idx = 0; idx < P; idx++) {
        uint64_t plane_size = uint64_t(ceil(double(G - begin) / (P - idx)));
        // k: first index with cgood[k] == cgood[begin] + plane_size (or n)
        const uint64_t remaining = uint64_t(cgood[n]) - uint64_t(cgood[begin]);
        uint64_t lo = begin, hi = uint64_t(n);
        if (plane_size > remaining) {
            lo = uint64_t(n);
        } else {
            const uint64_t target = uint64_t(cgood[begin]) + plane_size;
            while (lo < hi) {
                uint64_t mid = (lo + hi) / 2;
                if (uint64_t(cgood[mid]) >= target)
                    hi = mid;
                else
                    lo = mid + 1;
            }
        }
        first[idx] = int64_t(begin);
        last[idx] = int64_t(lo);
        begin = lo;
    }
    (void)absw_sorted;
    (void)median;
}

// One block per plane: plane w = mean |w| over good visibilities (or the
// median rule), in the plane's sorted range.
__global__ void k_wplane_values(const uint32_t* cgood, const double* absw_sorted, const uint8_t* good_sorted,
    const int64_t* first, const int64_t* last, int64_t n, int P, int median, double* w_avg)
{
    const int p = blockIdx.x;
    const int64_t b = first[p], e = last[p];
    __shared__ double s[256];
    if (!median) {
        double t = 0.0;
        for (int64_t k = b + threadIdx.x; k < e; k += blockDim.x)
            if (good_sorted[k])
                t += absw_sorted[k];
        s[threadIdx.x] = t;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o)
                s[threadIdx.x] += s[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            uint64_t cnt = uint64_t(cgood[e]) - uint64_t(cgood[b]);
            w_avg[p] = cnt > 0 ? s[0] / double(cnt) : 0.0;
        }
    } else if (threadIdx.x == 0) {
        // median variant (gridder.cpp:79-118)
        const uint64_t G = cgood[n];
        uint64_t plane_size = uint64_t(ceil(double(G - uint64_t(b)) / (P - p)));
        uint64_t middle = plane_size / 2;
        if (uint64_t(b) + plane_size > G)
            middle = (G - uint64_t(b)) / 2;
        uint64_t counter = uint64_t(cgood[e]) - uint64_t(cgood[b]);
        if (counter == 0) {
            w_avg[p] = 0.0;
            return;
        }
        // idx_mid: position of the (middle)-th good from b
        uint64_t target = uint64_t(cgood[b]) + middle; // cgood[k] == target and good[k]
        int64_t lo = b, hi = e;
        while (lo < hi) {
            int64_t mid = (lo + hi) / 2;
            if (uint64_t(cgood[mid + 1]) > target)
                hi = mid;
            else
                lo = mid + 1;
        }
        int64_t idx_mid = lo;
        if ((plane_size % 2) == 0 && idx_mid > 0)
            w_avg[p] = (absw_sorted[idx_mid - 1] + absw_sorted[idx_mid]) / 2.0;
        else
            w_avg[p] = absw_sorted[idx_mid];
    }
}

// Mean |w| per plane in two deterministic steps: block b sums the good |w|
// of its slice [b*chunk, (b+1)*chunk) of the sorted array separately for
// every plane the slice meets (partial[p][b]); then one block per plane adds
// its partials in block order.
__global__ void __launch_bounds__(256) k_wplane_partial(const double* __restrict__ absw_sorted,
    const uint8_t* __restrict__ good_sorted, const int64_t* first, const int64_t* last, int64_t n, int P,
    int64_t chunk, int nblk, double* partial)
{
    __shared__ double red[256];
    const int64_t a = int64_t(blockIdx.x) * chunk;
    const int64_t b = min(n, a + chunk);
    if (a >= b)
        return;
    int p = 0;
    {
        int lo = 0, hi = P - 1; // last plane with first <= a
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (first[mid] <= a)
                lo = mid;
            else
                hi = mid - 1;
        }
        p = lo;
    }
    for (; p < P && first[p] < b; p++) {
        const int64_t s0 = max(a, first[p]), s1 = min(b, last[p]);
        double t = 0.0;
#pragma unroll 2
        for (int64_t k = s0 + threadIdx.x; k < s1; k += blockDim.x)
            if (good_sorted[k])
                t += absw_sorted[k];
        red[threadIdx.x] = t;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o)
                red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0)
            partial[int64_t(p) * nblk + blockIdx.x] = red[0];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_wplane_finish(const double* partial, const uint32_t* cgood,
    const int64_t* first, const int64_t* last, int64_t chunk, int nblk, double* w_avg)
{
    __shared__ double red[256];
    const int p = blockIdx.x;
    const int64_t f = first[p], l = last[p];
    double t = 0.0;
    if (l > f) {
        const int b0 = int(f / chunk), b1 = int((l - 1) / chunk);
        for (int bb = b0 + int(threadIdx.x); bb <= b1; bb += blockDim.x)
            t += partial[int64_t(p) * nblk + bb];
    }
    red[threadIdx.x] = t;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const uint64_t cnt = uint64_t(cgood[l]) - uint64_t(cgood[f]);
        w_avg[p] = cnt > 0 ? red[0] / double(cnt) : 0.0;
    }
}

template <typename R>
__global__ void k_gather_good(const uint32_t* perm, const Item<R>* items, const double* absw, int64_t n,
    uint8_t* good_sorted, uint32_t* gflag, double* absw_sorted, Item<R>* items_sorted)
{
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const uint32_t i = perm[k];
    const Item<R> it = items[i];
    uint8_t g = it.good != 0;
    good_sorted[k] = g;
    gflag[k] = g;
    if (absw_sorted)
        absw_sorted[k] = absw[i];
    if (items_sorted)
        items_sorted[k] = it; // binning and gridding read the items in |w| order
}

// ---------------------------------------------------------------- W-planes without the |w| sort
//
// The reference's W-planes (gridder.cpp:68-146) take equal counts of the
// |w|-sorted visibilities.  When every visibility is good, plane p holds the
// sorted ranks [G_p, G_p+1) with G_0 = 0, G_p+1 = G_p + ceil((n - G_p) / (P -
// p)), so an item's plane follows from how many plane-start items precede
// it in the sort order ((|w| bits, input index), the stable order).  Those
// P - 1 items are found without sorting: a histogram of the 24-bit keys'
// top 12 bits (k_wsel_hist) places each start rank in a bin and at a rank
// within it (k_wsel_plan); the members of those bins are collected
// (k_wsel_collect) and each start item is the member of its bin with the
// wanted rank under the exact order (k_wsel_resolve: every member counts the
// members before it).  k_wsel_classify then gives every item its plane (a
// binary search over the start items) and sums |w| per plane exactly, in
// 64-bit fixed point relative to the plane's smallest |w| (so the sums do
// not depend on the order of the additions); k_wsel_finish forms the means
// and plane starts.  Items not all good, non-finite |w|, more than WSEL_MAXP
// planes or a start bin of more than WSEL_CAP members set bit 16 of the
// error word: the host then runs the sorting path.
constexpr int WSEL_BINS_LOG = 16;
constexpr int WSEL_BINS = 1 << WSEL_BINS_LOG; // key24 >> 8
constexpr int WSEL_CAP = 2048;  // members of a start item's bin that k_wsel_resolve holds
constexpr int WSEL_MAXP = 1024; // planes

struct WselState {
    // zeroed before the pass
    uint32_t hist[WSEL_BINS];
    uint32_t cursor[WSEL_MAXP];
    unsigned long long sum[WSEL_MAXP];
    // written by k_wsel_plan / k_wsel_resolve
    int32_t binmap[WSEL_BINS];      // list of a start bin, -1 otherwise
    uint32_t list_off[WSEL_MAXP + 1];
    uint32_t list_cnt[WSEL_MAXP];
    int32_t start_list[WSEL_MAXP];  // per plane p >= 1: its start item's list
    uint32_t start_rank[WSEL_MAXP]; // and rank within the list's bin
    uint32_t start_bin[WSEL_MAXP];
    uint32_t chunk_tot[1024];       // bins per 64-bin chunk (k_wsel_chunks)
    unsigned long long start_bits[WSEL_MAXP]; // the start item: |w| bits, input index
    uint32_t start_idx[WSEL_MAXP];
    int64_t G[WSEL_MAXP + 1];
    int valid;
};
constexpr size_t kWselZeroWords = (sizeof(uint32_t) * (WSEL_BINS + WSEL_MAXP) + sizeof(unsigned long long) * WSEL_MAXP) / 4;

// (the keys of k_wkey24, formed here and again in k_wsel_collect from |w|)
__global__ void __launch_bounds__(256) k_wsel_hist(const double* __restrict__ absw, int64_t n, const double* total,
    WselState* ws)
{
    const WKey kf(total, n);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        atomicAdd(&ws->hist[kf(absw[i]) >> (24 - WSEL_BINS_LOG)], 1u);
    // no start bins yet (k_wsel_plan marks them)
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < WSEL_BINS; b += gridDim.x * blockDim.x)
        ws->binmap[b] = -1;
}

// Exclusive scan over the 1024 threads of a block of the values v; *total =
// their sum.
__device__ __forceinline__ uint32_t wsel_block_scan(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t wsum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o)
                w += y;
        }
        wsum[lane] = w; // inclusive over the warps
    }
    __syncthreads();
    const uint32_t r = x - v + (warp ? wsum[warp - 1] : 0u);
    *total = wsum[31];
    __syncthreads();
    return r;
}

// Totals of the 1024 chunks of 64 bins, one warp a chunk (coalesced).
__global__ void __launch_bounds__(1024) k_wsel_chunks(WselState* ws)
{
    const int c = blockIdx.x * 32 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    const uint2 v = reinterpret_cast<const uint2*>(ws->hist + 64 * c)[lane];
    uint32_t t = v.x + v.y;
    for (int o = 16; o > 0; o >>= 1)
        t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0)
        ws->chunk_tot[c] = t;
}

// One block of 1024 threads.  The plane starts have a closed form: with q =
// n / P and r = n % P, ceil((n - G_p) / (P - p)) = q + [p < r], so G_p = p q +
// min(p, r).  A block scan of the chunk totals (k_wsel_chunks) locates each
// start rank's chunk, and the plane's thread walks the chunk's 64 bins to the
// bin and the rank within it.  The start bins become lists in plane order.
__global__ void __launch_bounds__(1024) k_wsel_plan(WselState* ws, int64_t n, int P, const unsigned long long* ngood,
    unsigned int* err)
{
    constexpr int PER = WSEL_BINS / 1024;
    __shared__ uint32_t chunk[1025]; // prefix at each thread's first bin
    const int tid = threadIdx.x;
    const bool ok0 = ngood[0] == (unsigned long long)n && P >= 1 && P <= WSEL_MAXP;
    const uint32_t t = ws->chunk_tot[tid];
    uint32_t total = 0;
    const uint32_t excl = wsel_block_scan(t, &total);
    chunk[tid] = excl;
    if (tid == 0)
        chunk[1024] = total;
    const int64_t qn = P >= 1 ? n / P : 0, rn = P >= 1 ? n % P : 0;
    auto G = [&](int p) { return int64_t(p) * qn + (int64_t(p) < rn ? int64_t(p) : rn); };
    if (ok0)
        for (int p = tid; p <= P; p += blockDim.x)
            ws->G[p] = G(p);
    __syncthreads();
    // plane p = tid: its start item's bin (the last b whose prefix is <= G_p)
    // and rank within it, and the bin's size
    const int p = tid;
    const bool has = ok0 && p >= 1 && p < P && G(p) < n;
    uint32_t bin = 0, m = 0;
    if (has) {
        const uint32_t gp = uint32_t(G(p));
        int lo = 0, hi = 1023;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (chunk[mid] <= gp)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint4* c4 = reinterpret_cast<const uint4*>(ws->hist + PER * lo);
        uint32_t before = chunk[lo];
        bool found = false;
        for (int q = 0; q < PER / 4 && !found; q++) {
            const uint4 v = c4[q];
            const uint32_t w[4] = { v.x, v.y, v.z, v.w };
            for (int e = 0; e < 4; e++) {
                if (before + w[e] > gp) { // rank gp lies in this bin
                    bin = uint32_t(PER * lo + 4 * q + e);
                    m = w[e];
                    found = true;
                    break;
                }
                before += w[e];
            }
        }
        ws->start_bin[p] = bin;
        ws->start_rank[p] = gp - before;
    }
    __shared__ uint32_t sbin[1024];
    __shared__ int bad;
    sbin[tid] = bin;
    if (tid == 0)
        bad = !ok0;
    __syncthreads();
    // a start bin opens a list unless the previous plane's start is in it
    const bool opens = has && !(p >= 2 && G(p - 1) < n && sbin[p - 1] == bin);
    if (opens && m > uint32_t(WSEL_CAP))
        bad = 1;
    uint32_t nlist = 0, noff = 0;
    const uint32_t li = wsel_block_scan(opens ? 1u : 0u, &nlist);
    const uint32_t off = wsel_block_scan(opens ? m : 0u, &noff);
    __shared__ uint32_t slist[1024];
    slist[tid] = opens ? li : 0u;
    __syncthreads();
    if (bad) {
        if (tid == 0) {
            ws->valid = 0;
            atomicOr(err, 16u);
        }
        return;
    }
    if (opens) {
        ws->binmap[bin] = int32_t(li);
        ws->list_off[li] = off;
        ws->list_cnt[li] = m;
    }
    if (p >= 1 && p < P) {
        // the list of this plane's start: that of the last plane up to p that
        // opened one (planes after the items run out have none)
        int32_t l = -1;
        if (has) {
            int q = p;
            while (q >= 2 && G(q - 1) < n && sbin[q - 1] == bin)
                q--;
            l = int32_t(slist[q]);
        }
        ws->start_list[p] = l;
    }
    if (tid == 0) {
        ws->list_off[nlist] = noff;
        ws->valid = 1;
    }
}

__global__ void __launch_bounds__(256) k_wsel_collect(const double* __restrict__ absw, int64_t n, const double* total,
    WselState* ws, unsigned long long* mbits, uint32_t* midx)
{
    if (!ws->valid)
        return;
    const WKey kf(total, n);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const double a = absw[i];
        const int li = ws->binmap[kf(a) >> (24 - WSEL_BINS_LOG)];
        if (li >= 0) {
            const uint32_t pos = ws->list_off[li] + atomicAdd(&ws->cursor[li], 1u);
            mbits[pos] = __double_as_longlong(a);
            midx[pos] = uint32_t(i);
        }
    }
}

// One block per plane p >= 1: the member of the start item's bin whose rank
// under (|w| bits, index) is the wanted one.
__global__ void __launch_bounds__(256) k_wsel_resolve(WselState* ws, const unsigned long long* mbits, const uint32_t* midx)
{
    __shared__ unsigned long long sb[WSEL_CAP];
    __shared__ uint32_t si[WSEL_CAP];
    const int p = blockIdx.x + 1;
    if (!ws->valid)
        return;
    const int li = ws->start_list[p];
    if (li < 0) {
        if (threadIdx.x == 0) {
            ws->start_bits[p] = ~0ull; // after every item: the plane and all later ones are empty
            ws->start_idx[p] = ~0u;
        }
        return;
    }
    const uint32_t off = ws->list_off[li], m = ws->list_cnt[li], want = ws->start_rank[p];
    for (uint32_t e = threadIdx.x; e < m; e += blockDim.x) {
        sb[e] = mbits[off + e];
        si[e] = midx[off + e];
    }
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < m; e += blockDim.x) {
        const unsigned long long b = sb[e];
        const uint32_t ix = si[e];
        uint32_t r = 0;
        for (uint32_t f = 0; f < m; f++)
            r += (sb[f] < b || (sb[f] == b && si[f] < ix)) ? 1u : 0u;
        if (r == want) {
            ws->start_bits[p] = b;
            ws->start_idx[p] = ix;
        }
    }
}

// Plane p's smallest |w| (its start item's; 0 for plane 0) and the fixed-point
// scale of its sums: 2^e with (width * count) * 2^e <= 2^61, width = the
// plane's |w| range (up to the next start item, or wmax).
__device__ __forceinline__ void wsel_range(const WselState* ws, int p, int P, int64_t n, double wmax, double& lo,
    double& scale)
{
    const int64_t cnt = ws->G[p + 1] - ws->G[p];
    lo = p == 0 ? 0.0 : __longlong_as_double((long long)ws->start_bits[p]);
    const double hi = (p + 1 < P && ws->G[p + 1] < n) ? __longlong_as_double((long long)ws->start_bits[p + 1]) : wmax;
    const double span = (hi - lo) * double(cnt);
    if (cnt <= 0 || !(span > 0.0)) {
        scale = 1.0;
        return;
    }
    int ex;
    frexp(span, &ex); // span < 2^ex
    scale = ldexp(1.0, 61 - ex);
}

__global__ void __launch_bounds__(256) k_wsel_classify(const double* __restrict__ absw, int64_t n, int P,
    const double* total, WselState* ws, uint16_t* plane16, unsigned int* err)
{
    __shared__ unsigned long long sbits[WSEL_MAXP];
    __shared__ uint32_t sidx[WSEL_MAXP];
    __shared__ double slo[WSEL_MAXP], sscale[WSEL_MAXP];
    // the sums: one copy per warp when the planes fit (less contention on
    // the shared atomics), else one copy for the block
    __shared__ unsigned long long acc[WSEL_MAXP];
    constexpr int kWarpCopyP = WSEL_MAXP / 8;
    const int copies = P <= kWarpCopyP ? 8 : 1;
    if (!ws->valid) {
        // plane 0 for every item: the binning that follows stays in bounds
        // (the host grids again on the sorting path)
        for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
            plane16[i] = 0;
        return;
    }
    const double wmax = total[1];
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        sbits[p] = p == 0 ? 0ull : ws->start_bits[p];
        sidx[p] = p == 0 ? 0u : ws->start_idx[p];
        wsel_range(ws, p, P, n, wmax, slo[p], sscale[p]);
    }
    for (int q = threadIdx.x; q < copies * P; q += blockDim.x)
        acc[q] = 0;
    __syncthreads();
    unsigned long long* myacc = acc + (copies > 1 ? ((threadIdx.x >> 5) & 7) * P : 0);
    bool bad = false;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
        const double a = absw[i];
        if (!(a <= wmax)) { // non-finite |w|
            plane16[i] = 0;
            bad = true;
            continue;
        }
        const unsigned long long b = __double_as_longlong(a);
        const uint32_t ix = uint32_t(i);
        // the last plane whose start item is at or before (b, ix)
        int lo = 0, hi = P - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (sbits[mid] < b || (sbits[mid] == b && sidx[mid] <= ix))
                lo = mid;
            else
                hi = mid - 1;
        }
        plane16[i] = uint16_t(lo);
        const double d = a - slo[lo];
        atomicAdd(&myacc[lo], (unsigned long long)rint(d * sscale[lo]));
    }
    if (bad)
        atomicOr(err, 16u);
    __syncthreads();
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        unsigned long long v = 0;
        for (int c = 0; c < copies; c++)
            v += acc[c * P + p];
        if (v)
            atomicAdd(&ws->sum[p], v);
    }
}

__global__ void __launch_bounds__(256) k_wsel_finish(const WselState* ws, int64_t n, int P, const double* total,
    double* w_avg, int64_t* first)
{
    if (!ws->valid) {
        for (int p = threadIdx.x; p < P; p += blockDim.x) {
            w_avg[p] = 0.0;
            first[p] = 0;
        }
        return;
    }
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
        double lo, scale;
        wsel_range(ws, p, P, n, total[1], lo, scale);
        const int64_t cnt = ws->G[p + 1] - ws->G[p];
        w_avg[p] = cnt > 0 ? lo + (double(ws->sum[p]) / scale) / double(cnt) : 0.0;
        first[p] = ws->G[p];
    }
}

// The |w| order from a stable sort on the 24-bit keys of k_wkey24 is exact
// except inside runs of equal keys, whose members are in index order.  Each
// run is re-sorted by the full 64-bit key (the bits of |w|), keeping index
// order among equal |w|: the result is the stable order of the 64-bit sort.  Runs longer than kFixRun whose |w| are not all equal set
// bit 4 of *err (the caller then repeats the step with the 64-bit sort).
constexpr int kFixRun = 32;
__global__ void k_fix_runs(const uint32_t* __restrict__ key32, uint32_t* perm, const unsigned long long* __restrict__ key64,
    int64_t n, unsigned int* err)
{
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k + 1 >= n)
        return;
    const uint32_t kk = key32[k];
    if ((k > 0 && key32[k - 1] == kk) || key32[k + 1] != kk)
        return; // not the start of a run of length >= 2
    int64_t e = k + 2;
    while (e < n && e - k <= kFixRun && key32[e] == kk)
        e++;
    const int len = int(e - k);
    if (len == 2) { // the common run: one compare, no per-thread arrays
        const uint32_t p0 = perm[k], p1 = perm[k + 1];
        if (key64[p1] < key64[p0]) {
            perm[k] = p1;
            perm[k + 1] = p0;
        }
        return;
    }
    if (len > kFixRun) {
        const unsigned long long first = key64[perm[k]];
        for (int64_t j = k + 1; j < n && key32[j] == kk; j++)
            if (key64[perm[j]] != first) {
                atomicOr(err, 4u);
                return;
            }
        return; // all |w| equal: index order is already the stable order
    }
    unsigned long long kv[kFixRun];
    uint32_t pv[kFixRun];
    for (int a = 0; a < len; a++) {
        pv[a] = perm[k + a];
        kv[a] = key64[pv[a]];
    }
    // insertion sort by (key64, index): stable, so equal keys keep index order
    for (int a = 1; a < len; a++) {
        const unsigned long long x = kv[a];
        const uint32_t y = pv[a];
        int b = a - 1;
        while (b >= 0 && kv[b] > x) {
            kv[b + 1] = kv[b];
            pv[b + 1] = pv[b];
            b--;
        }
        kv[b + 1] = x;
        pv[b + 1] = y;
    }
    for (int a = 0; a < len; a++)
        perm[k + a] = pv[a];
}

// W-kernel generation for one plane per CTA (FP64), the non-Hankel path of
// WideFieldImaging (aw_projection.cpp:50-111 image-domain kernel with
// combine_2d_kernel_value :455-474, forward c2c FFT :194, truncation
// :197-209, kernel cache :415-448).
//
// The image-domain kernel comb(a, b) is even in both indices (the reference
// writes each value at (+-a, +-b)), non-zero only for |a|, |b| < half, so its
// forward DFT is the separable cosine sum
//   conv(k, l) = sum_{a,b >= 0} m_a m_b Q[a][b] cos(2 pi k a / arr) cos(2 pi l b / arr)
// with m_0 = 1, m_{>0} = 2, and conv(+-k, +-l) = conv(|k|, |l|).  Only the
// entries the cache samples are formed: first the l = 0 row for the
// truncation, then the |offset| block of the truncated support.
// Outputs per plane: support, conv quadrant conv[p][l][k] (stride lh_max)
// and inv[p][y][x] = 1 / sum(Re) of each oversampled sub-kernel, so that the
// reference's cached kernel value is conv * inv.
struct WkParams {
    const double* w_avg;
    const double* aa; // image-domain AA kernel over the workarea
    const double* ctab; // cos(2 pi t / arr), t < arr
    int half, arr, os, cs, max_support, lh_max;
    int ctab_in_smem; // k_wkernel_plane: launched with arr doubles of dynamic shared memory
    double scaled_cell, trunc_perc;
    double2* Qs;   // scratch [P][half][half]
    double2* Ts;   // scratch [P][lh_max][half]
    double2* convd; // [P][lh_max][lh_max] FP64
    double* invd;   // [P][cs][cs]
    int* support;
};

__device__ __forceinline__ double2 wk_value(const WkParams& q, double w, int px, int py)
{
    const int half = q.half;
    const double dx = double(px) * q.scaled_cell, dy = double(py) * q.scaled_cell;
    const double r2 = dx * dx + dy * dy;
    if (r2 >= 1.0)
        return make_double2(q.aa[half + px] * q.aa[half + py], 0.0);
    const double nn = sqrt(1.0 - r2);
    const double ph = (-2.0 * 3.141592653589793238462643383279502884) * w * (nn - 1.0);
    double sn, cn;
    sincos(ph, &sn, &cn);
    const double re = (cn / nn) * q.aa[half + px];
    const double im = (sn / nn) * q.aa[half + px];
    return make_double2(re * q.aa[half + py], im * q.aa[half + py]);
}

// 1/sum(Re) of each oversampled sub-kernel of plane p (ty outer, tx inner as
// in generate_kernel_cache, aw_projection.cpp:383-448); conv is the plane's
// quadrant conv[|dy| * lh + |dx|].
__device__ void wk_inverse_sums(const WkParams& q, int p, const double2* conv, int S)
{
    const int cs = q.cs, os = q.os, lh = q.lh_max;
    const int K = 2 * S + 1;
    for (int t = threadIdx.x; t < cs * cs; t += blockDim.x) {
        const int x = t % cs, y = t / cs;
        double ks = 0.0;
        for (int j = 0; j < K; j++) {
            int ox = (j - S) * os + os / 2 - x;
            ox = ox < 0 ? -ox : ox;
            for (int i = 0; i < K; i++) {
                int oy = (i - S) * os + os / 2 - y;
                oy = oy < 0 ? -oy : oy;
                ks += conv[size_t(oy) * lh + ox].x;
            }
        }
        q.invd[(size_t(p) * cs + y) * cs + x] = 1 / ks;
    }
}

__global__ void __launch_bounds__(1024) k_wkernel_plane(WkParams q)
{
    const int p = blockIdx.x;
    const int half = q.half, arr = q.arr, os = q.os, lh = q.lh_max;
    const double w = q.w_avg[p];
    double2* Q = q.Qs + size_t(p) * half * half;
    double2* T = q.Ts + size_t(p) * lh * half;
    double2* conv = q.convd + size_t(p) * lh * lh;
    __shared__ double2 row0[1024];
    __shared__ int s_support;
    // the cosine table in shared memory when the launch gave room for it
    extern __shared__ double sct[];
    const double* ct = q.ctab;
    if (q.ctab_in_smem) {
        for (int t = threadIdx.x; t < arr; t += blockDim.x)
            sct[t] = q.ctab[t];
        ct = sct;
    }
    auto C = [&](int t) { return ct[t % arr]; };
    // 1. image-domain quadrant Q[a][b] (row a, column b)
    for (int t = threadIdx.x; t < half * half; t += blockDim.x) {
        const int a = t % half, b = t / half;
        double2 v;
        if (a == 0 && b == 0)
            v = make_double2(q.aa[half] * q.aa[half], 0.0);
        else if (b == 0)
            v = wk_value(q, w, a, 0);
        else if (a == 0)
            v = wk_value(q, w, b, 0); // output(0, i) reuses value(i, 0)
        else
            v = wk_value(q, w, a, b);
        Q[size_t(b) * half + a] = v;
    }
    __syncthreads();
    // 2. T[0][a] = sum_b m_b Q[a][b]
    for (int a = threadIdx.x; a < half; a += blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int b = 0; b < half; b++) {
            const double m = b == 0 ? 1.0 : 2.0;
            const double2 v = Q[size_t(b) * half + a];
            re += v.x * m;
            im += v.y * m;
        }
        T[a] = make_double2(re, im);
    }
    __syncthreads();
    // 3. conv(k, 0) at k = i*os for the truncation (k <= arr/2)
    const int kmax0 = min(q.max_support * os, arr >> 1);
    const int nrow = kmax0 / os + 1;
    for (int t = threadIdx.x; t < nrow && t < 1024; t += blockDim.x) {
        const int k = t * os;
        double re = 0.0, im = 0.0;
        for (int a = 0; a < half; a++) {
            const double c = (a == 0 ? 1.0 : 2.0) * C(k * a);
            re += T[a].x * c;
            im += T[a].y * c;
        }
        row0[t] = make_double2(re, im);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int S = q.max_support;
        if (q.trunc_perc > 0.0) {
            const double minv = hypot(row0[0].x, row0[0].y) * (q.trunc_perc / 100.0);
            unsigned i = unsigned(kmax0);
            while (i > 0) {
                const double2 v = row0[i / os];
                if (hypot(v.x, v.y) > minv)
                    break;
                i -= os;
            }
            S = int(min(unsigned(i / os), unsigned(q.max_support)));
        }
        s_support = S;
        q.support[p] = S;
    }
    __syncthreads();
    const int S = s_support;
    const int L = min(S * os + os / 2 + 1, (arr >> 1) + 1);
    // 4. T[l][a] for l < L
    for (int t = threadIdx.x; t < L * half; t += blockDim.x) {
        const int a = t % half, l = t / half;
        double re = 0.0, im = 0.0;
        for (int b = 0; b < half; b++) {
            const double c = (b == 0 ? 1.0 : 2.0) * C(l * b);
            const double2 v = Q[size_t(b) * half + a];
            re += v.x * c;
            im += v.y * c;
        }
        T[size_t(l) * half + a] = make_double2(re, im);
    }
    __syncthreads();
    // 5. conv(k, l) for k, l < L
    for (int t = threadIdx.x; t < L * L; t += blockDim.x) {
        const int k = t % L, l = t / L;
        double re = 0.0, im = 0.0;
        const double2* Tl = T + size_t(l) * half;
        for (int a = 0; a < half; a++) {
            const double c = (a == 0 ? 1.0 : 2.0) * C(k * a);
            re += Tl[a].x * c;
            im += Tl[a].y * c;
        }
        conv[size_t(l) * lh + k] = make_double2(re, im);
    }
    __syncthreads();
    wk_inverse_sums(q, p, conv, S);
}

// Hankel-transform W-kernels (hankel_opt, aw_projection.cpp:211-287 and
// RadialInterpolate, aw_projection.h:126-214): the radially symmetric W-kernel
// comes from a 1-D transform of the image-domain kernel's radial profile,
// interpolated at the radius of every kernel offset.
struct HankelParams {
    int n;          // radial samples: arr/2 (discrete Hankel transform) or arr (projection slice)
    int proj_slice; // hankel_proj_slice: 1-D DFT of the kernel's projection onto one axis
    int cubic;      // InterpType::CUBIC: natural cubic spline; otherwise linear
    double2* R;     // scratch [P][half]: radial profile or projection
    double2* Y;     // scratch [P][n]: transform at radii 0..n-1 (oversampled uv pixels)
    double2* B;     // scratch [P][n]: spline quadratic coefficients
    double* Cp;     // scratch [P][2][n]: forward-sweep factors of the spline solve
};

// Cubic (natural boundary, tk::spline semantics) or linear interpolation of
// the unit-spaced samples Y at radius r; k = min(floor(r), n - 1), beyond the
// last sample the end segment extrapolates linearly.
__device__ __forceinline__ double2 hankel_interp(const HankelParams& h, const double2* Y, const double2* B, double r)
{
    const int n = h.n;
    const int k = min(int(r), n - 1);
    const double t = r - double(k);
    const double2 y = Y[k];
    if (!h.cubic) {
        const double2 y0 = k < n - 1 ? y : Y[n - 2];
        const double2 y1 = k < n - 1 ? Y[k + 1] : Y[n - 1];
        return make_double2((y1.x - y0.x) * t + y.x, (y1.y - y0.y) * t + y.y);
    }
    auto coef = [&](int i, double2& a, double2& b, double2& c) { // segment i < n - 1
        const double2 b0 = B[i], b1 = B[i + 1], y0 = Y[i], y1 = Y[i + 1];
        a = make_double2(1.0 / 3.0 * (b1.x - b0.x), 1.0 / 3.0 * (b1.y - b0.y));
        b = b0;
        c = make_double2((y1.x - y0.x) - 1.0 / 3.0 * (2.0 * b0.x + b1.x),
                         (y1.y - y0.y) - 1.0 / 3.0 * (2.0 * b0.y + b1.y));
    };
    double2 a, b, c;
    if (k < n - 1) {
        coef(k, a, b, c);
    } else {
        // end segment: a = 0, b = b[n-1] (0 for the natural spline), c = derivative at the last node
        double2 a2, b2, c2;
        coef(n - 2, a2, b2, c2);
        a = make_double2(0.0, 0.0);
        b = B[n - 1];
        c = make_double2(3.0 * a2.x + 2.0 * b2.x + c2.x, 3.0 * a2.y + 2.0 * b2.y + c2.y);
    }
    return make_double2(((a.x * t + b.x) * t + c.x) * t + y.x, ((a.y * t + b.y) * t + c.y) * t + y.y);
}

// One block per W-plane.  Writes the plane's support, its quadrant
// conv[|dy| * lh + |dx|] = f(sqrt(dx^2 + dy^2)) and the sub-kernel
// normalisations, the same outputs as k_wkernel_plane.
__global__ void __launch_bounds__(1024) k_hankel_plane(WkParams q, HankelParams h)
{
    const int p = blockIdx.x;
    const int half = q.half, arr = q.arr, os = q.os, lh = q.lh_max, n = h.n;
    const double w = q.w_avg[p];
    double2* R = h.R + size_t(p) * half;
    double2* Y = h.Y + size_t(p) * n;
    double2* B = h.B + size_t(p) * n;
    double2* conv = q.convd + size_t(p) * lh * lh;
    __shared__ int s_support;
    constexpr double kPi = 3.141592653589793238462643383279502884;
    // 1. radial profile (aw_projection.cpp:226-240) or projection (:113-170)
    for (int j = threadIdx.x; j < half; j += blockDim.x) {
        double2 v;
        if (!h.proj_slice) {
            const double dx = double(j) * q.scaled_cell;
            const double r2 = dx * dx;
            if (r2 >= 1.0) {
                v = make_double2(q.aa[half + j], 0.0);
            } else {
                const double nn = sqrt(1.0 - r2);
                double sn, cn;
                sincos((-2.0 * kPi) * w * (nn - 1.0), &sn, &cn);
                v = make_double2((cn / nn) * q.aa[half + j], (sn / nn) * q.aa[half + j]);
            }
        } else if (j == 0) {
            double re = 0.0, im = 0.0;
            for (int i = 1; i < half; i++) {
                const double2 e = wk_value(q, w, i, 0);
                re += e.x;
                im += e.y;
            }
            v = make_double2(re * 2.0 + q.aa[half] * q.aa[half], im * 2.0);
        } else {
            v = wk_value(q, w, j, 0);
            for (int i = 1; i < half; i++) {
                const double2 e = wk_value(q, w, i, j);
                v.x += e.x * 2.0;
                v.y += e.y * 2.0;
            }
        }
        R[j] = v;
    }
    __syncthreads();
    // 2. transform at radii k < n
    const int jmax = min(half, n);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double re = 0.0, im = 0.0;
        if (!h.proj_slice) {
            // DHT column k (aw_projection.cpp:532-596): annulus j spans
            // [rn_{j-1}, rn_j], rn_j = j + 1/2 except rn_{n-1} = n - 1
            const double kk = (kPi / double(n)) * double(k);
            const double kn = (2.0 * kPi) / kk;
            double prev = 0.0;
            for (int j = 0; j < jmax; j++) {
                const double rn = j == n - 1 ? double(n - 1) : double(j) + 0.5;
                const double F = k == 0 ? kPi * rn * rn : kn * rn * besselj1_ref(kk * rn);
                const double d = j == 0 ? F : F - prev;
                prev = F;
                re += d * R[j].x;
                im += d * R[j].y;
            }
        } else {
            // length-arr DFT of the even projection (fft_fftw_dft_c2c_1d)
            re = R[0].x;
            im = R[0].y;
            for (int t = 1; t < half; t++) {
                const double c = 2.0 * q.ctab[(k * t) % arr];
                re += R[t].x * c;
                im += R[t].y * c;
            }
        }
        Y[k] = make_double2(re, im);
    }
    __syncthreads();
    // 3. truncation (aw_projection.h:135-148)
    if (threadIdx.x == 0) {
        int S = q.max_support;
        if (q.trunc_perc > 0.0) {
            const double minv = hypot(Y[0].x, Y[0].y) * (q.trunc_perc / 100.0);
            int t = q.max_support * os;
            while (t > n - 1)
                t -= os;
            while (t > os) {
                if (hypot(Y[t].x, Y[t].y) > minv)
                    break;
                t -= os;
            }
            S = min(int(ceil(double(t) * (1.0 / double(os)))), q.max_support);
        }
        s_support = S;
        q.support[p] = S;
    }
    // 4. natural cubic spline: b_0 = b_{n-1} = 0 and, for 0 < i < n-1,
    //    b_{i-1}/3 + 4 b_i/3 + b_{i+1}/3 = y_{i+1} - 2 y_i + y_{i-1}
    //    (tridiagonal, forward elimination and back substitution; real and
    //    imaginary parts in two threads)
    if (h.cubic && threadIdx.x < 2) {
        const int comp = threadIdx.x;
        const double* y = reinterpret_cast<const double*>(Y) + comp;
        double* b = reinterpret_cast<double*>(B) + comp;
        double* cp = h.Cp + (size_t(p) * 2 + comp) * n;
        b[0] = 0.0;
        b[2 * (n - 1)] = 0.0;
        double cprev = 0.0, dprev = 0.0;
        for (int i = 1; i <= n - 2; i++) {
            const double rhs = (y[2 * (i + 1)] - y[2 * i]) - (y[2 * i] - y[2 * (i - 1)]);
            const double m = 4.0 / 3.0 - (1.0 / 3.0) * cprev;
            cprev = (1.0 / 3.0) / m;
            dprev = (rhs - (1.0 / 3.0) * dprev) / m;
            cp[i] = cprev;
            b[2 * i] = dprev;
        }
        for (int i = n - 3; i >= 1; i--)
            b[2 * i] -= cp[i] * b[2 * (i + 1)];
    }
    __syncthreads();
    // 5. kernel quadrant at the radius of each offset
    const int S = s_support;
    const int L = min(S * os + os / 2 + 1, lh);
    for (int t = threadIdx.x; t < L * L; t += blockDim.x) {
        const int dx = t % L, dy = t / L;
        const double r = dy == 0 ? double(dx) : (dx == 0 ? double(dy) : sqrt(double(dx * dx + dy * dy)));
        conv[size_t(dy) * lh + dx] = hankel_interp(h, Y, B, r);
    }
    __syncthreads();
    wk_inverse_sums(q, p, conv, S);
}

__global__ void k_cos_table(int arr, double* c)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < arr)
        c[t] = cospi(2.0 * double(t) / double(arr));
}

// FP32 copies of the W-kernel tables for the single-precision gridders.
// Per-snapshot scalars of a batch, gathered for one read-back.
struct BatchScalars {
    double total;
    unsigned long long ngood;
    uint32_t nitems;
    uint32_t err;
    int32_t max_support;
    int32_t pad;
};

__global__ void k_collect_scalars(const double* total, const unsigned long long* ngood, const uint32_t* nitems,
    const unsigned int* err, const int* psup, int nplanes, BatchScalars* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    BatchScalars b;
    b.total = total[0];
    b.ngood = ngood[0];
    b.nitems = nitems[0];
    b.err = err[0];
    int m = 0;
    for (int p = 0; p < nplanes; p++)
        m = max(m, psup[p]);
    b.max_support = m;
    b.pad = 0;
    *out = b;
}

// Expanded W-kernel tables for the gridder: one block per (plane, oversampled
// offset pair); entry t = i*K + j holds the reference's cached kernel value
// conv(|oy|, |ox|) * inv (aw_projection.cpp:415-448), formed in FP64 and
// rounded once to R.  Plane p's tables start at off[p] = sum over q < p of
// cs^2 * K_q^2.
template <typename R>
__global__ void k_wk_expand(const double2* convd, const double* invd, const int* support, int P, int cs, int os,
    int lh, typename Cplx<R>::T* out, uint32_t* off)
{
    const int p = blockIdx.x;
    const int pair = blockIdx.y;
    const int cy = pair / cs, cx = pair % cs;
    uint32_t base = 0;
    for (int q = 0; q < p; q++) {
        const uint32_t Kq = uint32_t(2 * support[q] + 1);
        base += uint32_t(cs) * uint32_t(cs) * Kq * Kq;
    }
    if (pair == 0 && threadIdx.x == 0)
        off[p] = base;
    const int S = support[p];
    const int K = 2 * S + 1;
    const double inv = invd[(size_t(p) * cs + cy) * cs + cx];
    const double2* conv = convd + size_t(p) * lh * lh;
    typename Cplx<R>::T* dst = out + base + uint32_t(pair) * uint32_t(K * K);
    for (int t = threadIdx.x; t < K * K; t += blockDim.x) {
        const int i = t / K, j = t % K;
        int oy = (i - S) * os + os / 2 - cy;
        int ox = (j - S) * os + os / 2 - cx;
        oy = oy < 0 ? -oy : oy;
        ox = ox < 0 ? -ox : ox;
        const double2 v = conv[size_t(oy) * lh + ox];
        typename Cplx<R>::T o;
        o.x = R(v.x * inv);
        o.y = R(v.y * inv);
        dst[t] = o;
    }
}

// The scalars a call reads back, gathered for one copy: sampling-grid
// total, good visibilities, tile-list entries, error flags and the largest
// plane support (one warp).
struct ScalarPack {
    double total;
    unsigned long long ngood;
    uint32_t nitems;
    unsigned int err;
    int max_support;
    int pad;
};

// Copies of a call's results into page-locked host memory through its device
// address: the na words of a, then the 16-byte units of b that hold the
// first a[count_word] records of rec_bytes each (all nb units when
// count_word < 0), at most nb.
__global__ void k_copy_out(const uint32_t* a, uint32_t* ha, int na, const uint4* b, uint4* hb, int nb,
    int count_word, int rec_bytes)
{
    const int t = int(blockIdx.x * blockDim.x + threadIdx.x), stride = int(gridDim.x * blockDim.x);
    for (int i = t; i < na; i += stride)
        ha[i] = a[i];
    int n = nb;
    if (count_word >= 0)
        n = int(min((uint64_t(a[count_word]) * uint64_t(rec_bytes) + 15) / 16, uint64_t(nb)));
    for (int i = t; i < n; i += stride)
        hb[i] = b[i];
}

__global__ void k_pack_scalars(const double* total, const unsigned long long* ngood, const uint32_t* nitems,
    const unsigned int* err, const int* sup, int nsup, ScalarPack* out)
{
    int m = 0;
    for (int i = threadIdx.x; i < nsup; i += 32)
        m = max(m, sup[i]);
    for (int o = 16; o > 0; o >>= 1)
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) {
        out->total = *total;
        out->ngood = *ngood;
        out->nitems = *nitems;
        out->err = *err;
        out->max_support = m;
        out->pad = 0;
    }
}

} // namespace stpgpu
