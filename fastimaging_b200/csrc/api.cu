// Host orchestration and the extern "C" layer (include/stpgpu.h).
//
// One stpgpu_context = one device + one stream + cached scratch buffers and
// cuFFT plans.  An entry point enqueues its whole pipeline on the context
// stream and synchronises once at the end to read back the few scalars the
// caller needs.
#include <cub/cub.cuh>
#include <cufft.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <initializer_list>
#include <iterator>
#include <utility>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <unordered_map>
#include <chrono>
#include <thread>
#include <memory>
#include <deque>
#include <condition_variable>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "imager_kernels.cuh"
#include "sourcefind_kernels.cuh"
#include "visibility_kernels.cuh"
#include "aproj_kernels.cuh"

using namespace stpgpu;

namespace {
// Zeroes ranges of 32-bit words (at most four) with one kernel launch.
void zero_words(cudaStream_t st, std::initializer_list<std::pair<void*, int64_t>> ranges)
{
    ZeroRanges z {};
    int64_t most = 0;
    int r = 0;
    for (const auto& q : ranges) {
        z.p[r] = static_cast<uint32_t*>(q.first);
        z.n[r] = q.second;
        most = std::max(most, q.second);
        r++;
    }
    const unsigned blocks = unsigned(std::min<int64_t>(std::max<int64_t>((most + 255) / 256, 1), 148 * 4));
    k_zero_ranges<<<blocks, 256, 0, st>>>(z);
    STPGPU_CHECK_LAUNCH();
}

// A captured graph with its zero-filling memset nodes (the library's own
// scratch clears, e.g. CUB's) replaced by k_zero_ranges kernel nodes: a
// replayed graph spends 2-5 us of idle time at a memset node, about 0.1 us
// at a kernel node.  Works on a clone; returns the clone, or the original
// graph when a node cannot be rewritten (nothing is changed then);
// *added = the kernel nodes added.
cudaGraph_t memsets_to_kernels(cudaGraph_t graph, int* added)
{
    *added = 0;
    size_t count = 0;
    if (cudaGraphGetNodes(graph, nullptr, &count) != cudaSuccess || count == 0)
        return graph;
    cudaGraph_t clone = nullptr;
    if (cudaGraphClone(&clone, graph) != cudaSuccess)
        return graph;
    auto give_up = [&] {
        cudaGraphDestroy(clone);
        (void)cudaGetLastError();
        *added = 0;
        return graph;
    };
    std::vector<cudaGraphNode_t> nodes(count);
    if (cudaGraphGetNodes(clone, nodes.data(), &count) != cudaSuccess)
        return give_up();
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType type;
        if (cudaGraphNodeGetType(nd, &type) != cudaSuccess)
            return give_up();
        if (type != cudaGraphNodeTypeMemset)
            continue;
        cudaMemsetParams mp {};
        if (cudaGraphMemsetNodeGetParams(nd, &mp) != cudaSuccess)
            return give_up();
        const size_t bytes = size_t(mp.width) * mp.elementSize;
        if (mp.value != 0 || mp.height != 1 || bytes % 4 != 0 || (reinterpret_cast<uintptr_t>(mp.dst) & 3) != 0)
            continue;
        size_t nin = 0, nout = 0;
        if (cudaGraphNodeGetDependencies(nd, nullptr, &nin) != cudaSuccess
            || cudaGraphNodeGetDependentNodes(nd, nullptr, &nout) != cudaSuccess)
            return give_up();
        std::vector<cudaGraphNode_t> in(nin), out(nout);
        if ((nin && cudaGraphNodeGetDependencies(nd, in.data(), &nin) != cudaSuccess)
            || (nout && cudaGraphNodeGetDependentNodes(nd, out.data(), &nout) != cudaSuccess))
            return give_up();
        ZeroRanges z {};
        z.p[0] = static_cast<uint32_t*>(mp.dst);
        z.n[0] = int64_t(bytes / 4);
        void* args[] = { &z };
        cudaKernelNodeParams kp {};
        kp.func = reinterpret_cast<void*>(k_zero_ranges);
        kp.gridDim = dim3(unsigned(std::min<int64_t>(std::max<int64_t>((z.n[0] + 255) / 256, 1), 148 * 4)));
        kp.blockDim = dim3(256);
        kp.sharedMemBytes = 0;
        kp.kernelParams = args;
        cudaGraphNode_t kn = nullptr;
        if (cudaGraphAddKernelNode(&kn, clone, nin ? in.data() : nullptr, nin, &kp) != cudaSuccess)
            return give_up();
        for (cudaGraphNode_t o : out)
            if (cudaGraphAddDependencies(clone, &kn, &o, 1) != cudaSuccess)
                return give_up();
        if (cudaGraphDestroyNode(nd) != cudaSuccess)
            return give_up();
        ++*added;
    }
    cudaGraphDestroy(graph);
    return clone;
}
} // namespace

namespace {
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

// Device outputs of one gridding pass (context buffers).
struct GridOut {
    void* grid = nullptr;
    void* beam = nullptr;
    int image_rows = 0;
    double* d_total = nullptr;             // [0] sample_grid_total
    unsigned long long* d_ngood = nullptr; // [0] good visibilities
    uint32_t* d_nitems = nullptr;          // tile-list entries
    unsigned int* d_err = nullptr;
    int* d_plane_support = nullptr;
    int nplanes = 0;
};

} // namespace

struct stpgpu_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    bool timing = false;
    cudaEvent_t pev[5] = { nullptr, nullptr, nullptr, nullptr, nullptr };
    std::string err;

    void mark(int k)
    {
        if (timing && pev[k])
            STPGPU_CUDA_TRY(cudaEventRecord(pev[k], stream));
    }
    std::map<std::string, DevBuf> bufs;
    std::map<std::tuple<int, int, cudaStream_t>, cufftHandle> plans; // (N, cufftType, stream)
    std::map<std::tuple<int, int, int, cudaStream_t>, cufftHandle> plans_many; // (N, type, batch, stream)
    // Prefix of buffer and memo names: the batch path gives every snapshot
    // slot its own buffers ("b<i>/"); single calls use "".
    std::string ns;

    // batch path: worker streams, fork/join events, the captured graph of
    // the last batch signature, the tile-width choice per size class and a
    // pinned staging area (gridder parameter tables, scalar read-back)
    std::vector<cudaStream_t> wstreams;
    std::vector<cudaEvent_t> wevents;
    cudaEvent_t fork_ev = nullptr;
    std::string batch_sig;
    int batch_calls = 0;
    cudaGraph_t batch_graph = nullptr;
    cudaGraphExec_t batch_exec = nullptr;
    // gridder layouts chosen by the autotuner, per size class; shared by the
    // slot contexts of a server so that a class is tuned once
    struct TuneTable {
        std::mutex mu;
        std::map<std::string, int> m;
    };
    std::shared_ptr<TuneTable> tunes = std::make_shared<TuneTable>();
    bool tune_get(const std::string& k, int& v)
    {
        std::lock_guard<std::mutex> lk(tunes->mu);
        auto it = tunes->m.find(k);
        if (it == tunes->m.end())
            return false;
        v = it->second;
        return true;
    }
    void tune_set(const std::string& k, int v)
    {
        std::lock_guard<std::mutex> lk(tunes->mu);
        tunes->m[k] = v;
    }
    cudaEvent_t tev[2] = { nullptr, nullptr };
    void* batch_host = nullptr;
    size_t batch_host_cap = 0;

    // single-call path: graph of the last device-pointer call (see run_imager)
    std::string single_sig;
    cudaGraph_t single_graph = nullptr;
    cudaGraphExec_t single_exec = nullptr;
    GridOut single_g {};
    uint32_t sf_label_cap = 0; // source finder: label-analysis capacities that sufficed so far
    uint32_t sf_fg_cap = 0;
    int single_launches = 0; // our kernels in single_graph (counted at capture)
    int batch_launches = 0;  // our kernels in batch_graph
    // source finder: graph of the first attempt of the last call (see
    // run_source_find); sf_graph_off after a capture that failed
    std::string sf_sig;
    cudaGraph_t sf_graph = nullptr;
    cudaGraphExec_t sf_exec = nullptr;
    int sf_launches = 0;
    bool sf_graph_off = false;
    // size classes whose last single call could not take the W-planes
    // without the |w| sort (their calls sort)
    std::set<std::string> wsel_off;
    // bumped whenever a device buffer or the page-locked stage is
    // reallocated: a captured graph whose signature holds an older value
    // may point at freed memory
    uint64_t buf_gen = 0;

    void drop_sf_graph()
    {
        if (sf_exec)
            cudaGraphExecDestroy(sf_exec);
        if (sf_graph)
            cudaGraphDestroy(sf_graph);
        sf_exec = nullptr;
        sf_graph = nullptr;
        sf_sig.clear();
    }

    void drop_single()
    {
        if (single_exec)
            cudaGraphExecDestroy(single_exec);
        if (single_graph)
            cudaGraphDestroy(single_graph);
        single_exec = nullptr;
        single_graph = nullptr;
        single_sig.clear();
    }

    void drop_graph()
    {
        if (batch_exec)
            cudaGraphExecDestroy(batch_exec);
        if (batch_graph)
            cudaGraphDestroy(batch_graph);
        batch_exec = nullptr;
        batch_graph = nullptr;
    }
    void* pinned = nullptr;
    void* pinned_dev = nullptr; // the device's address of the staging area (mapped)
    size_t pinned_cap = 0;
    std::map<std::string, std::string> memo_keys; // buffer name -> key of its current contents
    // staged gridder: records per visibility last counted, per namespace,
    // tile width, support and truncation (absent: count at the next call)
    std::map<std::string, double> rec_ratio;

    // True when buffer `name` already holds the data described by `key`
    // (static tables: gcf, kernel tables, cos tables); records `key`.
    bool memo(const std::string& name, const std::string& key)
    {
        auto it = memo_keys.find(ns + name);
        if (it != memo_keys.end() && it->second == key)
            return true;
        memo_keys[ns + name] = key;
        return false;
    }

    // STPGPU_LOG_ALLOC=1: one line per allocation or plan creation with its
    // host time (allocations after warm-up are what stall a serving loop)
    static void log_alloc(const char* what, const std::string& name, size_t bytes,
        std::chrono::steady_clock::time_point t0)
    {
        static const bool on = std::getenv("STPGPU_LOG_ALLOC") != nullptr;
        if (!on)
            return;
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "stpgpu alloc: %s %s %zu bytes %.3f ms\n", what, name.c_str(), bytes, ms);
    }

    // Named scratch buffer, grown on demand (steady state allocates nothing).
    template <typename T>
    T* buf(const std::string& name, size_t count)
    {
        const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
        DevBuf& b = bufs[ns + name];
        if (b.cap < bytes) {
            if (b.p) {
                STPGPU_CUDA_TRY(cudaStreamSynchronize(stream));
                STPGPU_CUDA_TRY(cudaFree(b.p));
                b.p = nullptr;
                b.cap = 0;
            }
            const size_t want = bytes + bytes / 8;
            const auto t0 = std::chrono::steady_clock::now();
            buf_gen++;
            STPGPU_CUDA_TRY(cudaMalloc(&b.p, want));
            log_alloc("device buffer", ns + name, want, t0);
            b.cap = want;
            memo_keys.erase(ns + name);
        }
        return reinterpret_cast<T*>(b.p);
    }

    template <typename T>
    T* host_stage(size_t count)
    {
        const size_t bytes = std::max<size_t>(count * sizeof(T), 256);
        if (pinned_cap < bytes) {
            if (pinned) {
                STPGPU_CUDA_TRY(cudaStreamSynchronize(stream));
                cudaFreeHost(pinned);
            }
            pinned = nullptr;
            pinned_dev = nullptr;
            pinned_cap = 0;
            const auto t0 = std::chrono::steady_clock::now();
            buf_gen++;
            STPGPU_CUDA_TRY(cudaHostAlloc(&pinned, bytes, cudaHostAllocMapped));
            STPGPU_CUDA_TRY(cudaHostGetDevicePointer(&pinned_dev, pinned, 0));
            log_alloc("page-locked stage", ns, bytes, t0);
            pinned_cap = bytes;
        }
        return reinterpret_cast<T*>(pinned);
    }

    // The device's address of a location in the staging area: kernels write
    // a call's results there directly (a kernel node in place of a copy node
    // in the captured graphs).
    template <typename T>
    T* host_stage_dev(T* h) const
    {
        return reinterpret_cast<T*>(static_cast<unsigned char*>(pinned_dev)
            + (reinterpret_cast<unsigned char*>(h) - static_cast<unsigned char*>(pinned)));
    }

    // One plan per (size, type, stream): a plan's work area must not be
    // shared by transforms running concurrently on different streams.
    cufftHandle plan(int N, cufftType type)
    {
        const auto key = std::make_tuple(N, int(type), stream);
        auto it = plans.find(key);
        if (it != plans.end())
            return it->second;
        cufftHandle h;
        const auto t0 = std::chrono::steady_clock::now();
        cufftResult r = cufftPlan2d(&h, N, N, type);
        log_alloc("cuFFT plan", ns + "N" + std::to_string(N), 0, t0);
        if (r != CUFFT_SUCCESS)
            fail(STPGPU_ERR_CUFFT, "cufftPlan2d failed (" + std::to_string(int(r)) + ") for N=" + std::to_string(N));
        r = cufftSetStream(h, stream);
        if (r != CUFFT_SUCCESS)
            fail(STPGPU_ERR_CUFFT, "cufftSetStream failed");
        plans[key] = h;
        return h;
    }

    // Batched N x N transforms (A-projection kernels), cached like plan().
    cufftHandle plan_many(int N, cufftType type, int batch)
    {
        const auto key = std::make_tuple(N, int(type), batch, stream);
        auto it = plans_many.find(key);
        if (it != plans_many.end())
            return it->second;
        cufftHandle h;
        int dims[2] = { N, N };
        const auto t0 = std::chrono::steady_clock::now();
        cufftResult r = cufftPlanMany(&h, 2, dims, nullptr, 1, N * N, nullptr, 1, N * N, type, batch);
        log_alloc("cuFFT plan", ns + "N" + std::to_string(N) + "x" + std::to_string(batch), 0, t0);
        if (r != CUFFT_SUCCESS)
            fail(STPGPU_ERR_CUFFT, "cufftPlanMany failed (" + std::to_string(int(r)) + ") for N=" + std::to_string(N));
        r = cufftSetStream(h, stream);
        if (r != CUFFT_SUCCESS)
            fail(STPGPU_ERR_CUFFT, "cufftSetStream failed");
        plans_many[key] = h;
        return h;
    }

    void release()
    {
        if (stream)
            cudaStreamSynchronize(stream);
        for (auto w : wstreams)
            cudaStreamSynchronize(w);
        drop_graph();
        drop_single();
        drop_sf_graph();
        batch_sig.clear();
        batch_calls = 0;
        for (auto& kv : plans)
            cufftDestroy(kv.second);
        plans.clear();
        for (auto& kv : plans_many)
            cufftDestroy(kv.second);
        plans_many.clear();
        for (auto& kv : bufs)
            if (kv.second.p)
                cudaFree(kv.second.p);
        bufs.clear();
        memo_keys.clear();
    }
};

namespace {

std::string fkey(double v)
{
    char b[64];
    std::snprintf(b, sizeof(b), "%a", v);
    return b;
}

constexpr size_t pad256(size_t b) { return (b + 255) / 256 * 256; }

inline unsigned grid1d(int64_t n, int threads) { return unsigned(std::max<int64_t>(1, ceil_div(n, threads))); }

stpgpu_status guard(stpgpu_context* ctx, const std::function<void()>& f)
{
    if (!ctx)
        return STPGPU_ERR_INVALID_ARG;
    try {
        STPGPU_CUDA_TRY(cudaSetDevice(ctx->device));
        f();
        ctx->err.clear();
        return STPGPU_OK;
    } catch (const Error& e) {
        ctx->err = e.msg;
        if (ctx->stream)
            cudaStreamSynchronize(ctx->stream);
        return e.status;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return STPGPU_ERR_CUDA;
    }
}

double arc_sec_to_rad(double v) { return (v / 3600.0) * (M_PI / 180.0); } // gridder.h:20

// ------------------------------------------------------------------ imager

struct ImagerSetup {
    int kf = kPSWF;
    double trunc = 0.0; // functor argument
    int support = 0;    // AA kernel support
    int N = 0;          // padded (grid) size
    int kernel_exact = 0;
    int os = 1;
    int shift_uv = 1, halfplane = 1, beam = 0;
    int analytic = 0;
    double cell_size = 0.0;
    int nplanes = 0, max_support = 0, undersampling = 1, wmedian = 0;
    double trunc_perc = 0.0;
    int full_wsort = 0; // |w| order from the 64-bit sort (fallback of the 32-bit sort + run fix-up)
    int wsel = 0;       // W-planes without the |w| sort (k_wsel_*; single calls, falls back through error bit 16)
    int hankel = 0, proj_slice = 0, cubic = 0; // Hankel-transform W-kernels (hankel_opt)
    // A-projection: time steps, rotated-kernel option, pointing (radians),
    // per-visibility hour angles (device pointer once the call has staged
    // them) and the beam's spherical-harmonic coefficients (host)
    int ntimesteps = 0, aproj_opt = 0;
    double obs_dec = 0.0, obs_ra = 0.0;
    const double* lha = nullptr;
    const double* pbcoefs = nullptr;
    int npbcoefs = 0;
    // compensated FP32 only: grid cells stored in double and the c2r done in
    // double precision (wide_fft_needed decides)
    int wide_fft = 0;
};

// W-projection with a maximum support above 32: the W-kernel tables and tile
// lists are sized from the measured plane supports and list length (two
// host round trips) instead of from the worst case, so such calls are not
// captured into CUDA graphs.
bool large_support(const ImagerSetup& s) { return s.nplanes > 0 && s.max_support > 32; }

void check_pars(const ImagerSetup& s)
{
    if (s.N <= 0 || (s.N % 2) != 0)
        fail(STPGPU_ERR_INVALID_ARG, "grid size must be a positive even number");
    if (s.support <= 0)
        fail(STPGPU_ERR_INVALID_ARG, "kernel_support must be > 0");
    if (s.nplanes > 0 && s.max_support <= 0)
        fail(STPGPU_ERR_INVALID_ARG, "max_wpconv_support must be > 0 with W-projection");
    if (s.nplanes > 65535)
        fail(STPGPU_ERR_INVALID_ARG, "num_wplanes too large");
    if (s.nplanes > 0 && s.max_support > 127)
        fail(STPGPU_ERR_UNSUPPORTED, "max_wpconv_support > 127 is outside the GPU path");
    if (s.nplanes == 0 && s.support > 32)
        fail(STPGPU_ERR_UNSUPPORTED, "kernel_support > 32 is outside the GPU path");
    if (s.os > 4096)
        fail(STPGPU_ERR_INVALID_ARG, "oversampling too large");
}

// Key of the tile autotuner: calls of one class share the tile width.
std::string size_class(const ImagerSetup& s, int precision)
{
    const int conv = s.nplanes > 0 ? s.max_support : s.support;
    // W-projection: the truncation percentage decides the plane supports, so it is part of the class
    return "p" + std::to_string(precision) + "/k" + std::to_string(s.nplanes > 0 ? 2 : (s.kernel_exact ? 1 : 0))
        + "/N" + std::to_string(s.N) + "/S" + std::to_string(conv) + "/os" + std::to_string(s.os)
        + (s.nplanes > 0 ? "/t" + fkey(s.trunc_perc) : std::string());
}

// Gridder launch prepared by run_gridder when the caller launches it itself
// (the batch path merges the tiles of many snapshots into one launch).
enum GridKind { GK_NONE = 0, GK_SEP, GK_EXACT, GK_WPROJ };
template <typename R>
struct GridLaunch {
    int kind = GK_NONE;
    int beam = 0;
    int form = 0; // gridder form the binning was built for (0 lanes-per-item, 2 lane-per-tap, 3 staged)
    int tile_c = TILE_C_DEFAULT;
    int ntiles = 0;
    size_t smem = 0;
    GridParams<R> gp {};
};

// convolve_to_grid (gridder.h:240-997): grids into context buffers "grid"
// and "beamgrid" of precision R (complex), image_rows x N column-major.
// tile_c: grid columns per tile (32 or 16).  With `defer` the gridder kernel
// is not launched: its parameters are returned there instead.
// Autotuned gridder layout bits beside the tile width (low 8 bits).
constexpr int kLayoutPersist = 1 << 8; // batch: persistent work queue
constexpr int kLayoutCols = 1 << 9;    // column-packed tile gridder (grid_tile_cols)
constexpr int kLayoutTaps = 1 << 10;   // lane-per-tap tile gridder (grid_tile_taps)
constexpr int kLayoutRecs = 1 << 11;   // staged tile gridder over decoded records (grid_tile_recs)
// gridder form of a layout: 0 lanes-per-item, 1 column-packed, 2 lane-per-tap
// (3: staged records)
inline int form_of(int lay)
{
    return (lay & kLayoutRecs) ? 3 : ((lay & kLayoutCols) ? 1 : ((lay & kLayoutTaps) ? 2 : 0));
}

template <typename R, int COMP>
GridOut run_gridder(stpgpu_context* c, const ImagerSetup& s, const void* d_vis, int vis_c64, const double* d_wts,
    const double* d_uv, int uv_is_pixels, int64_t n, int tile_c = TILE_C_DEFAULT, GridLaunch<R>* defer = nullptr,
    int form = 0)
{
    if (tile_c != 32 && tile_c != 16 && !(tile_c == 8 && (form == 2 || form == 3)))
        fail(STPGPU_ERR_INVALID_ARG, "tile width must be 16 or 32 (8 with the lane-per-tap or staged gridder)");
    using C2 = typename Cplx<R>::T;
    check_pars(s);
    cudaStream_t st = c->stream;
    GridOut g;
    const int N = s.N;
    const bool wproj = s.nplanes > 0;
    const int conv_support = wproj ? s.max_support : s.support;
    const int kernel_exact = wproj ? 0 : s.kernel_exact;
    int os = s.os;
    if (kernel_exact) {
        os = 1;
    } else {
        os = (os >> 1) << 1;
        if (os == 0)
            os = 1;
    }
    const int cs = (os / 2) * 2 + 1;
    const int image_rows = s.halfplane ? N / 2 + 1 : N;
    g.image_rows = image_rows;
    const int64_t nn = std::max<int64_t>(n, 1);
    c->mark(0);

    // ---- prepass (gridder.h:369-423, :504)
    Item<R>* items = c->buf<Item<R>>("items", nn);
    const unsigned nb_pre = grid1d(n, GRID_THREADS);
    double* wpart = c->buf<double>("wpart", nb_pre);
    unsigned long long* npart = c->buf<unsigned long long>("npart", nb_pre);
    g.d_total = c->buf<double>("total", 4);
    g.d_ngood = c->buf<unsigned long long>("ngood", 2);
    g.d_err = c->buf<unsigned int>("err", 2);
    zero_words(st, { { g.d_err, 1 } });
    PrepassParams pp {};
    pp.n = n;
    pp.vis = d_vis;
    pp.vis_c64 = vis_c64;
    pp.weights = d_wts;
    pp.uv = d_uv;
    pp.uv_is_pixels = uv_is_pixels;
    pp.inv_px = arc_sec_to_rad(s.cell_size) * double(N); // imager.h:293
    pp.N = N;
    pp.conv_support = conv_support;
    pp.halfplane = s.halfplane;
    pp.shift_uv = s.shift_uv;
    pp.kernel_exact = kernel_exact;
    pp.os = os;
    pp.keep_w = wproj ? 1 : 0;
    pp.frac = kernel_exact ? c->buf<double>("frac", 2 * nn) : nullptr;
    pp.wsum_part = wpart;
    pp.ngood_part = npart;
    pp.absw_key = wproj ? c->buf<double>("absw", nn) : nullptr;
    pp.wmax_part = (wproj && !s.full_wsort) ? c->buf<double>("wmaxpart", 2 * size_t(nb_pre)) : nullptr;
    pp.iota = (wproj && !s.wsel) ? c->buf<uint32_t>("perm_in", nn) : nullptr;
    pp.w_out = nullptr;
    if (n > 0) {
        k_prepass<R><<<nb_pre, GRID_THREADS, 0, st>>>(pp, items);
        STPGPU_CHECK_LAUNCH();
    }
    k_finish_wsum<<<1, 1024, 0, st>>>(wpart, npart, pp.wmax_part, n > 0 ? int(nb_pre) : 0, g.d_total, g.d_ngood);
    STPGPU_CHECK_LAUNCH();

    // ---- kernels
    const uint32_t* sorted_perm = nullptr;
    Item<R>* items_sorted = nullptr; // W-projection: the items in |w| order
    const int64_t* plane_first = nullptr;
    int nplanes = 0;
    const R* k1d = nullptr;
    const C2* wconv = nullptr;
    const R* winv = nullptr;
    int lh = 0;
    C2* wk = nullptr;
    uint32_t* wk_off = nullptr;
    uint8_t* ts_of = nullptr; // A-projection time step per visibility
    int* plane_support = nullptr;
    if (!wproj && !kernel_exact) {
        // populate_kernel_cache (gridder.h:73-105) as a 1-D table, FP64 on the device
        const int K = 2 * s.support + 1;
        const std::string key = std::to_string(s.kf) + "/" + fkey(s.trunc) + "/" + std::to_string(s.support)
            + "/" + std::to_string(os);
        double* t64 = c->buf<double>("k1d64", size_t(cs) * K);
        if (!c->memo("k1d64", key)) {
            k_kernel_table<<<grid1d(cs, 64), 64, 0, st>>>(s.kf, s.trunc, s.support, os, t64);
            STPGPU_CHECK_LAUNCH();
        }
        if (sizeof(R) == 8) {
            k1d = reinterpret_cast<const R*>(t64);
        } else {
            float* t32 = c->buf<float>("k1d32", size_t(cs) * K);
            if (!c->memo("k1d32", key)) {
                k_d2f<<<grid1d(int64_t(cs) * K, 256), 256, 0, st>>>(t64, t32, int64_t(cs) * K);
                STPGPU_CHECK_LAUNCH();
            }
            k1d = reinterpret_cast<const R*>(t32);
        }
    }
    const uint16_t* plane16 = nullptr;
    if (wproj && n > 0 && s.wsel) {
        // the planes without sorting (k_wsel_*, see imager_kernels.cuh); a
        // condition it cannot meet sets error bit 16 and the caller grids
        // again on the sorting path
        const int P = s.nplanes;
        const unsigned g2 = std::min<unsigned>(grid1d(n, 256), 148 * 8);
        WselState* ws = c->buf<WselState>("wsel", 1);
        zero_words(st, { { ws, int64_t(kWselZeroWords) } });
        k_wsel_hist<<<std::min<unsigned>(grid1d(n, 256), 148 * 4), 256, 0, st>>>(pp.absw_key, n, g.d_total, ws);
        STPGPU_CHECK_LAUNCH();
        static_assert(WSEL_BINS == 1024 * 64, "chunks of 64 bins, 32 a block");
        k_wsel_chunks<<<32, 1024, 0, st>>>(ws);
        STPGPU_CHECK_LAUNCH();
        k_wsel_plan<<<1, 1024, 0, st>>>(ws, n, P, g.d_ngood, g.d_err);
        STPGPU_CHECK_LAUNCH();
        // members of the start bins: at most P - 1 bins of WSEL_CAP
        unsigned long long* mbits = c->buf<unsigned long long>("wsel_mb", size_t(std::max(P - 1, 1)) * WSEL_CAP);
        uint32_t* midx = c->buf<uint32_t>("wsel_mi", size_t(std::max(P - 1, 1)) * WSEL_CAP);
        k_wsel_collect<<<g2, 256, 0, st>>>(pp.absw_key, n, g.d_total, ws, mbits, midx);
        STPGPU_CHECK_LAUNCH();
        if (P > 1) {
            k_wsel_resolve<<<P - 1, 256, 0, st>>>(ws, mbits, midx);
            STPGPU_CHECK_LAUNCH();
        }
        uint16_t* pl = c->buf<uint16_t>("wsel_plane", nn);
        k_wsel_classify<<<g2, 256, 0, st>>>(pp.absw_key, n, P, g.d_total, ws, pl, g.d_err);
        STPGPU_CHECK_LAUNCH();
        int64_t* first = c->buf<int64_t>("pfirst", P);
        double* w_avg = c->buf<double>("wavg", P);
        k_wsel_finish<<<1, 256, 0, st>>>(ws, n, P, g.d_total, w_avg, first);
        STPGPU_CHECK_LAUNCH();
        plane16 = pl;
        plane_first = first;
        nplanes = P;
    } else if (wproj && n > 0) {
        const int P = s.nplanes;
        // |w| order (gridder.h:311-367): stable radix sort of 24-bit keys of
        // |w| (k_wkey24; three digit passes instead of the eight of the 64-bit
        // sort), then runs of equal keys re-sorted by the full |w| bits; with
        // full_wsort the IEEE bits of |w| themselves are sorted (64-bit keys;
        // non-negative doubles order as their bit patterns).
        const unsigned long long* keys64 = reinterpret_cast<const unsigned long long*>(pp.absw_key);
        uint32_t* perm_in = pp.iota;
        uint32_t* perm = c->buf<uint32_t>("perm", nn);
        size_t tb = 0;
        if (s.full_wsort) {
            unsigned long long* k64out = c->buf<unsigned long long>("absw64_sorted", nn);
            cub::DeviceRadixSort::SortPairs(nullptr, tb, keys64, k64out, perm_in, perm, int(n), 0, 64, st);
            void* tmp = c->buf<unsigned char>("cubtmp", tb);
            if (cub::DeviceRadixSort::SortPairs(tmp, tb, keys64, k64out, perm_in, perm, int(n), 0, 64, st)
                != cudaSuccess)
                fail(STPGPU_ERR_CUDA, "radix sort failed");
        } else {
            uint32_t* key24 = c->buf<uint32_t>("absw24", nn);
            k_wkey24<<<std::min<unsigned>(grid1d(n, 256), 148 * 8), 256, 0, st>>>(pp.absw_key, n, g.d_total, key24);
            STPGPU_CHECK_LAUNCH();
            uint32_t* k32out = c->buf<uint32_t>("absw24_sorted", nn);
            cub::DeviceRadixSort::SortPairs(nullptr, tb, key24, k32out, perm_in, perm, int(n), 0, 24, st);
            void* tmp = c->buf<unsigned char>("cubtmp", tb);
            if (cub::DeviceRadixSort::SortPairs(tmp, tb, key24, k32out, perm_in, perm, int(n), 0, 24, st)
                != cudaSuccess)
                fail(STPGPU_ERR_CUDA, "radix sort failed");
            k_fix_runs<<<grid1d(n, 256), 256, 0, st>>>(k32out, perm, keys64, n, g.d_err);
            STPGPU_CHECK_LAUNCH();
        }
        uint8_t* good_sorted = c->buf<uint8_t>("good_sorted", nn);
        uint32_t* gflag = c->buf<uint32_t>("gflag", nn + 1);
        uint32_t* cgood = c->buf<uint32_t>("cgood", nn + 1);
        double* absw_sorted = c->buf<double>("absw_sorted", nn);
        // binning and gridding read the items in |w| order (sequential
        // passes instead of gathers through the permutation)
        items_sorted = c->buf<Item<R>>("items_sorted", nn);
        k_gather_good<R><<<grid1d(n, 256), 256, 0, st>>>(perm, items, pp.absw_key, n, good_sorted, gflag, absw_sorted,
            items_sorted);
        STPGPU_CHECK_LAUNCH();
        zero_words(st, { { gflag + n, 1 } });
        size_t tb2 = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb2, gflag, cgood, int(n + 1), st);
        void* tmp2 = c->buf<unsigned char>("cubtmp2", tb2);
        if (cub::DeviceScan::ExclusiveSum(tmp2, tb2, gflag, cgood, int(n + 1), st) != cudaSuccess)
            fail(STPGPU_ERR_CUDA, "scan failed");
        int64_t* first = c->buf<int64_t>("pfirst", P);
        int64_t* last = c->buf<int64_t>("plast", P);
        double* w_avg = c->buf<double>("wavg", P);
        k_wplanes<<<1, 1, 0, st>>>(cgood, absw_sorted, n, P, s.wmedian, first, last);
        STPGPU_CHECK_LAUNCH();
        if (s.wmedian) {
            k_wplane_values<<<P, 256, 0, st>>>(cgood, absw_sorted, good_sorted, first, last, n, P, 1, w_avg);
            STPGPU_CHECK_LAUNCH();
        } else {
            const int nblk = int(std::min<int64_t>(2048, ceil_div(n, 512)));
            const int64_t chunk = ceil_div(n, nblk);
            double* partial = c->buf<double>("wpartial", size_t(P) * nblk);
            k_wplane_partial<<<nblk, 256, 0, st>>>(absw_sorted, good_sorted, first, last, n, P, chunk, nblk, partial);
            STPGPU_CHECK_LAUNCH();
            k_wplane_finish<<<P, 256, 0, st>>>(partial, cgood, first, last, chunk, nblk, w_avg);
            STPGPU_CHECK_LAUNCH();
        }
        sorted_perm = perm;
        plane_first = first;
        nplanes = P;
    }
    if (wproj && n > 0) {
        const int P = s.nplanes;
        double* w_avg = c->buf<double>("wavg", P); // the plane means, from either path above
        // W-kernels in FP64 (WideFieldImaging, aw_projection.cpp:19-111,173-210,366-452)
        const int K = 2 * s.max_support + 1;
        const int u = s.undersampling > 0 ? int(std::pow(2, s.undersampling - 1)) : 0;
        int workarea = 2;
        if (u > 0) {
            while ((workarea / u) < K)
                workarea *= 2;
        } else {
            while (workarea < N)
                workarea *= 2;
        }
        if (workarea < K)
            fail(STPGPU_ERR_INVALID_ARG, "W-kernel workarea smaller than the kernel size");
        const double scaling = double(N) / double(workarea);
        const int arr = workarea * os;
        if (arr % 2)
            fail(STPGPU_ERR_INVALID_ARG, "array_size must be multiple of 2 for WideFieldImaging generation.");
        if (int64_t(arr) * arr > (int64_t(1) << 31))
            fail(STPGPU_ERR_UNSUPPORTED, "W-kernel array too large");
        const int half = workarea / 2;
        const int Lh = std::min(s.max_support * os + os / 2 + 1, arr / 2 + 1);
        double* aa = c->buf<double>("aa", workarea);
        if (!c->memo("aa", std::to_string(s.kf) + "/" + fkey(s.trunc) + "/" + std::to_string(workarea) + "/"
                               + std::to_string(s.analytic))) {
            // ImgDomKernel(kernel_creator, workarea) (gridder.h:486)
            const int centre = workarea / 2;
            const int dmax = int(std::floor(s.trunc)) + 1;
            double ssum = 0.0;
            for (int d = -std::min(dmax, centre); d <= std::min(dmax, workarea - centre - 1); d++)
                ssum += kernel_value(s.kf, s.trunc, double(d));
            const double ksum_inv = ssum > 0.0 ? 1.0 / ssum : 1.0;
            k_imgdom_kernel<<<grid1d(workarea, 128), 128, 0, st>>>(s.kf, s.trunc, workarea, s.analytic, ksum_inv,
                dmax, aa);
            STPGPU_CHECK_LAUNCH();
        }
        double* ctab = c->buf<double>("ctab", arr);
        if (!c->memo("ctab", std::to_string(arr))) {
            k_cos_table<<<grid1d(arr, 256), 256, 0, st>>>(arr, ctab);
            STPGPU_CHECK_LAUNCH();
        }
        WkParams wq {};
        wq.w_avg = w_avg;
        wq.aa = aa;
        wq.ctab = ctab;
        wq.half = half;
        wq.arr = arr;
        wq.os = os;
        wq.cs = cs;
        wq.max_support = s.max_support;
        wq.lh_max = Lh;
        // WideFieldImaging gets real_t(arc_sec_to_rad(cell)), scaled by N/workarea
        wq.scaled_cell = arc_sec_to_rad(s.cell_size) * scaling;
        wq.trunc_perc = s.trunc_perc;
        if (!s.hankel) {
            wq.Qs = c->buf<double2>("wkQ", size_t(P) * half * half);
            wq.Ts = c->buf<double2>("wkT", size_t(P) * Lh * half);
        }
        wq.convd = c->buf<double2>("wkconv", size_t(P) * Lh * Lh);
        wq.invd = c->buf<double>("wkinv", size_t(P) * cs * cs);
        const int T = std::max(s.ntimesteps, 1);
        const int PT = P * T;
        plane_support = c->buf<int>("psupport", PT);
        wq.support = plane_support;
        const double2* aconv = nullptr; // A-projection: transformed kernels [P*T][arr][arr]
        if (s.ntimesteps > 0) {
            // time steps and their parallactic angles (gridder.h:507-520, gridder.cpp:148-200)
            double* iv = c->buf<double>("ap_iv", T + 1);
            double* lmean = c->buf<double>("ap_lmean", T);
            double* angle = c->buf<double>("ap_angle", T);
            ts_of = c->buf<uint8_t>("ap_ts", nn);
            k_lha_intervals<<<1, 1024, 0, st>>>(s.lha, n, T, iv);
            STPGPU_CHECK_LAUNCH();
            k_lha_steps<R><<<grid1d(n, 256), 256, 0, st>>>(s.lha, items, n, T, iv, ts_of);
            STPGPU_CHECK_LAUNCH();
            k_lha_means<R><<<T, 256, 0, st>>>(s.lha, items, ts_of, n, lmean);
            STPGPU_CHECK_LAUNCH();
            k_parangle<<<1, 256, 0, st>>>(lmean, T, s.obs_dec, s.obs_ra, angle);
            STPGPU_CHECK_LAUNCH();
            // inverse primary beam per step (one unrotated beam with aproj_opt)
            double* coefs = c->buf<double>("ap_coefs", s.npbcoefs);
            STPGPU_CUDA_TRY(
                cudaMemcpyAsync(coefs, s.pbcoefs, sizeof(double) * s.npbcoefs, cudaMemcpyHostToDevice, st));
            const int deg = (s.npbcoefs - 1) / 2;
            const double fov = arc_sec_to_rad(s.cell_size) * double(N);
            const int nA = s.aproj_opt ? 1 : T;
            double* Abeam = c->buf<double>("ap_beam", size_t(nA) * workarea * workarea);
            k_aproj_beam<<<grid1d(int64_t(nA) * workarea * workarea, 256), 256, 0, st>>>(nA, workarea, fov, coefs, deg,
                s.aproj_opt ? nullptr : angle, Abeam);
            STPGPU_CHECK_LAUNCH();
            // W-screen x beam, 2-D FFT per (plane, step) or per plane
            const int G = P * nA;
            const size_t img = size_t(arr) * arr;
            const size_t nimg = size_t(G) + (s.aproj_opt ? size_t(PT) : 0);
            if (nimg * img * sizeof(double2) > (uint64_t(8) << 30))
                fail(STPGPU_ERR_UNSUPPORTED,
                    "A-projection kernels exceed 8 GB (planes x time steps x (workarea x oversampling)^2)");
            double2* abuf = c->buf<double2>("ap_fft", nimg * img);
            STPGPU_CUDA_TRY(cudaMemsetAsync(abuf, 0, sizeof(double2) * size_t(G) * img, st));
            const int span = 2 * half - 1;
            k_aproj_screen<<<grid1d(int64_t(G) * span * span, 256), 256, 0, st>>>(wq, P, nA, Abeam, abuf);
            STPGPU_CHECK_LAUNCH();
            if (cufftExecZ2Z(c->plan_many(arr, CUFFT_Z2Z, G), reinterpret_cast<cufftDoubleComplex*>(abuf),
                    reinterpret_cast<cufftDoubleComplex*>(abuf), CUFFT_FORWARD)
                != CUFFT_SUCCESS)
                fail(STPGPU_ERR_CUFFT, "A-projection kernel FFT failed");
            k_aproj_support<<<grid1d(G, 128), 128, 0, st>>>(abuf, G, arr, os, s.max_support, s.trunc_perc,
                s.aproj_opt ? T : 1, plane_support);
            STPGPU_CHECK_LAUNCH();
            aconv = abuf;
            if (s.aproj_opt) {
                // rotate each plane's kernel by the step's angle, step after
                // step on the previous step's result (gridder.h:732-737)
                double2* rot = abuf + size_t(G) * img; // [P][T][arr][arr]
                for (int t = 0; t < T; t++) {
                    const double2* src = t == 0 ? abuf : rot + size_t(t - 1) * img;
                    const int64_t src_stride = t == 0 ? int64_t(img) : int64_t(T) * int64_t(img);
                    k_aproj_rotate<<<grid1d(int64_t(P) * int64_t(img), 256), 256, 0, st>>>(src, src_stride,
                        rot + size_t(t) * img, int64_t(T) * int64_t(img), P, arr, angle, t);
                    STPGPU_CHECK_LAUNCH();
                }
                aconv = rot;
            }
        } else if (s.hankel) {
            HankelParams hq {};
            hq.n = s.proj_slice ? arr : arr / 2;
            if (hq.n < 3)
                fail(STPGPU_ERR_INVALID_ARG, "Hankel transform needs more than 2 radial samples");
            hq.proj_slice = s.proj_slice;
            hq.cubic = s.cubic;
            hq.R = c->buf<double2>("hkR", size_t(P) * half);
            hq.Y = c->buf<double2>("hkY", size_t(P) * hq.n);
            hq.B = c->buf<double2>("hkB", size_t(P) * hq.n);
            hq.Cp = c->buf<double>("hkC", size_t(P) * 2 * hq.n);
            k_hankel_plane<<<P, 1024, 0, st>>>(wq, hq);
        } else {
            const size_t ct_bytes = sizeof(double) * size_t(arr);
            wq.ctab_in_smem = ct_bytes <= 24 * 1024;
            k_wkernel_plane<<<P, 1024, wq.ctab_in_smem ? ct_bytes : 0, st>>>(wq);
        }
        STPGPU_CHECK_LAUNCH();
        // per-offset K x K tables in the gridder's precision: worst-case
        // capacity (every plane at the maximum support), or with large
        // supports the sum over the measured plane supports
        uint64_t cap_wk = uint64_t(PT) * cs * cs * uint64_t(K) * K;
        if (large_support(s)) {
            std::vector<int> sup(PT);
            STPGPU_CUDA_TRY(cudaMemcpyAsync(sup.data(), plane_support, sizeof(int) * PT, cudaMemcpyDeviceToHost, st));
            STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
            cap_wk = 0;
            for (int v : sup)
                cap_wk += uint64_t(cs) * cs * uint64_t(2 * v + 1) * uint64_t(2 * v + 1);
            cap_wk = std::max<uint64_t>(cap_wk, 1);
        }
        if (cap_wk * sizeof(C2) > (uint64_t(16) << 30) || cap_wk > 0xffffffffull)
            fail(STPGPU_ERR_UNSUPPORTED, "W-kernel tables exceed 16 GB (planes x oversampling^2 x support^2)");
        wk = c->buf<C2>("wkexp", cap_wk);
        wk_off = c->buf<uint32_t>("wkoff", PT);
        if (aconv)
            k_aproj_expand<R><<<dim3(PT, cs * cs), 256, 0, st>>>(aconv, arr, plane_support, cs, os, wk, wk_off);
        else
            k_wk_expand<R><<<dim3(P, cs * cs), 64, 0, st>>>(wq.convd, wq.invd, plane_support, P, cs, os, Lh, wk,
                wk_off);
        STPGPU_CHECK_LAUNCH();
        lh = Lh;
        g.d_plane_support = plane_support;
        g.nplanes = PT;
    }

    const int kind = (wproj && n > 0) ? GK_WPROJ : (kernel_exact ? GK_EXACT : (!wproj ? GK_SEP : GK_NONE));
    // the clipped forms need one footprint segment per axis and tile
    const bool clip_ok = kind != GK_EXACT && N >= 2 * (2 * conv_support + 1 + 32) + 2;
    // staged records: tabulated kernels, no beam (else the lane-per-tap form)
    // and four warps' shared memory within the 227 KB of a block
    const size_t rec_wb = sizeof(Acc<R, COMP>) * TILE_R * size_t(tile_c) + 2 * kRecChunk * sizeof(TapRec<R>) + 16
        + (kind == GK_SEP ? sizeof(R) * size_t(cs) * size_t(2 * s.support + 1) : 0);
    const bool use_recs = form == 3 && clip_ok && !s.beam && (kind == GK_WPROJ || kind == GK_SEP)
        && 4 * (rec_wb + 15) <= 227 * 1024;
    if (form == 3 && !use_recs)
        form = 2;
    // 8-column tiles exist for the clipped lane-per-tap and staged forms only
    if (tile_c == 8 && !(clip_ok && (form == 2 || form == 3)))
        tile_c = 16;

    // ---- binning into 32x32 uv tiles
    const int tiles_r = int(ceil_div(image_rows, TILE_R));
    const int tiles_c = int(ceil_div(N, tile_c));
    const int ntiles = tiles_r * tiles_c;
    uint32_t* tcount = c->buf<uint32_t>("tcount", ntiles + 1);
    uint32_t* toff = c->buf<uint32_t>("toff", ntiles + 1);
    uint32_t* tcur = c->buf<uint32_t>("tcur", ntiles + 1);
    const int Kx = 2 * conv_support + 1;
    const uint64_t per_dim = uint64_t(ceil_div(Kx - 1, std::min(TILE_R, tile_c))) + 2;
    uint64_t cap = std::max<uint64_t>(1, uint64_t(nn) * 2 * per_dim * per_dim);
    if (!large_support(s) && cap > 0xffffffffull)
        fail(STPGPU_ERR_INVALID_ARG, "too many visibilities for one snapshot");
    uint32_t* list = (large_support(s) || use_recs) ? nullptr : c->buf<uint32_t>("tlist", cap);
    Item<R>* bin_items = items_sorted ? items_sorted : items;
    BinParams bp {};
    bp.plane16 = plane16;
    bp.N = N;
    bp.image_rows = image_rows;
    bp.tiles_r = tiles_r;
    bp.tiles_c = tiles_c;
    bp.tile_c = tile_c;
    bp.support = s.support;
    bp.plane_support = plane_support;
    bp.ts_of = ts_of;
    bp.ntimesteps = std::max(s.ntimesteps, 1);
    bp.exact = kernel_exact;
    bp.n = n;
    bp.tile_count = tcount;
    bp.tile_off = toff;
    bp.tile_cursor = tcur;
    // list slots kept by the count pass (the fill then needs no atomics)
    bp.ranks = c->buf<uint32_t>("tranks", size_t(std::max<int64_t>(n, 1)) * 2 * kRankSlots);
    bp.rank_overflow = c->buf<uint32_t>("trankovf", 1);
    bp.list = list;
    bp.list_capacity = cap;
    bp.err = g.d_err;
    zero_words(st, { { tcount, ntiles + 1 }, { tcur, ntiles + 1 }, { bp.rank_overflow, 1 } });
    if (n > 0) {
        k_count_tiles<R><<<grid1d(n, 256), 256, 0, st>>>(bp, bin_items, sorted_perm, plane_first, nplanes);
        STPGPU_CHECK_LAUNCH();
    }
    if (ntiles <= 4096) {
        k_scan_single<<<1, 1024, 0, st>>>(tcount, toff, ntiles);
        STPGPU_CHECK_LAUNCH();
    } else {
        // many tiles: the multi-block scan (tcount[ntiles] is 0, so
        // toff[ntiles] receives the total)
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, tcount, toff, ntiles + 1, st);
        void* tmp = c->buf<unsigned char>("cubtmp_tiles", tb);
        if (cub::DeviceScan::ExclusiveSum(tmp, tb, tcount, toff, ntiles + 1, st) != cudaSuccess)
            fail(STPGPU_ERR_CUDA, "tile offset scan failed");
        g_launches += 2;
    }
    TapRec<R>* recs = nullptr;
    uint64_t rec_cap = 0;
    if (use_recs) {
        // records sized from the records per visibility counted on the first
        // call of this namespace and class (one host round trip), scaled by
        // the call's visibilities with a quarter spare; a call that exceeds
        // the capacity sets bit 8 and the caller grids again after a fresh
        // count
        const std::string rkey = c->ns + "/" + std::to_string(tile_c) + "/S" + std::to_string(conv_support) + "/t"
            + fkey(s.trunc_perc) + "/os" + std::to_string(os);
        auto it = c->rec_ratio.find(rkey);
        if (it == c->rec_ratio.end() || large_support(s)) {
            uint32_t total = 0;
            STPGPU_CUDA_TRY(cudaMemcpyAsync(&total, toff + ntiles, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
            const double r = double(total) / double(nn);
            it = c->rec_ratio.insert_or_assign(rkey, it == c->rec_ratio.end() ? r : std::max(r, it->second)).first;
        }
        rec_cap = uint64_t(std::ceil(double(nn) * it->second * 1.25)) + 1024;
        recs = c->buf<TapRec<R>>("trecs", rec_cap);
        if (n > 0) {
            RecFill<R> rf { recs, rec_cap, wk_off, cs, os };
            if (kind == GK_WPROJ)
                k_fill_recs<R, KM_WPROJ><<<grid1d(n, 256), 256, 0, st>>>(bp, bin_items, sorted_perm, plane_first,
                    nplanes, rf);
            else
                k_fill_recs<R, KM_SEP><<<grid1d(n, 256), 256, 0, st>>>(bp, bin_items, sorted_perm, plane_first,
                    nplanes, rf);
            STPGPU_CHECK_LAUNCH();
        }
    } else {
        if (large_support(s)) { // size the list from the counted entries
            uint32_t total = 0;
            STPGPU_CUDA_TRY(cudaMemcpyAsync(&total, toff + ntiles, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
            cap = std::max<uint64_t>(total, 1);
            list = c->buf<uint32_t>("tlist", cap);
            bp.list = list;
            bp.list_capacity = cap;
        }
        if (n > 0) {
            k_fill_tiles<R><<<grid1d(n, 256), 256, 0, st>>>(bp, bin_items, sorted_perm, plane_first, nplanes);
            STPGPU_CHECK_LAUNCH();
        }
    }
    g.d_nitems = toff + ntiles;

    // ---- tile gridding
    // a wide grid (compensated FP32 for a double-precision c2r) holds double2 cells
    const int wide = (COMP == 1 && s.wide_fft) ? 1 : 0;
    const size_t cells = size_t(image_rows) * N * (wide ? 2 : 1);
    C2* grid = c->buf<C2>("grid", cells);
    C2* beam = s.beam ? c->buf<C2>("beamgrid", cells) : nullptr;
    GridParams<R> gp {};
    gp.N = N;
    gp.image_rows = image_rows;
    gp.tiles_r = tiles_r;
    gp.support = s.support;
    gp.os = os;
    gp.cs = cs;
    gp.exact_wrap = kernel_exact;
    gp.items = bin_items;
    gp.tile_off = toff;
    gp.list = list;
    gp.k1d = k1d;
    gp.kf = s.kf;
    gp.trunc = s.trunc;
    gp.frac = pp.frac;
    gp.n = n;
    gp.wconv = wconv;
    gp.winv = winv;
    gp.lh = lh;
    gp.plane_support = plane_support;
    gp.wk = wk;
    gp.wk_off = wk_off;
    gp.recs = recs;
    gp.rec_cap = rec_cap;
    gp.err = g.d_err;
    gp.grid = grid;
    gp.beam = beam;
    gp.wide = wide;
    using A = Acc<R, COMP>;
    size_t smem = size_t(TILE_R) * tile_c * sizeof(A) * (s.beam ? 2 : 1);
    if (!wproj && !kernel_exact)
        smem += sizeof(R) * size_t(cs) * (2 * s.support + 1);
    if (2 * conv_support + 1 > 255)
        fail(STPGPU_ERR_UNSUPPORTED, "kernel support > 127 is outside the GPU path");
    if (kind == GK_NONE) {
        STPGPU_CUDA_TRY(cudaMemsetAsync(grid, 0, sizeof(C2) * cells, st));
        if (beam)
            STPGPU_CUDA_TRY(cudaMemsetAsync(beam, 0, sizeof(C2) * cells, st));
    }
    if (defer) {
        defer->kind = kind;
        defer->beam = s.beam ? 1 : 0;
        defer->form = use_recs ? 3 : (form == 2 && clip_ok && kind != GK_EXACT ? 2 : 0);
        defer->tile_c = tile_c;
        defer->ntiles = kind == GK_NONE ? 0 : ntiles;
        defer->smem = use_recs ? (rec_wb + 15) / 16 * 16 : smem;
        defer->gp = gp;
    } else if (kind != GK_NONE) {
        auto launch = [&](auto kern) {
            if (smem > 48 * 1024)
                STPGPU_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            c->mark(1);
            kern<<<ntiles, 32, smem, st>>>(gp);
            STPGPU_CHECK_LAUNCH();
            c->mark(2);
        };
        const bool b = s.beam != 0;
        const bool t32 = tile_c == 32;
        const bool use_cols = form == 1 && clip_ok, use_taps = form == 2 && clip_ok;
        if (use_recs) {
            // four warps per block, each on its own tile
            const int sep_len = kind == GK_SEP ? cs * (2 * s.support + 1) : 0;
            auto launch_recs = [&](auto kern, size_t wb) {
                const size_t bs = 4 * wb;
                if (bs > 48 * 1024)
                    STPGPU_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bs)));
                c->mark(1);
                kern<<<unsigned((ntiles + 3) / 4), 128, bs, st>>>(gp, ntiles, int(wb));
                STPGPU_CHECK_LAUNCH();
                c->mark(2);
            };
            if (kind == GK_WPROJ) {
                if (tile_c == 8)
                    launch_recs(k_grid_tiles_recs<R, COMP, KM_WPROJ, 8, 4>, rec_warp_bytes<R, COMP, 8>(0));
                else if (tile_c == 16)
                    launch_recs(k_grid_tiles_recs<R, COMP, KM_WPROJ, 16, 4>, rec_warp_bytes<R, COMP, 16>(0));
                else
                    launch_recs(k_grid_tiles_recs<R, COMP, KM_WPROJ, 32, 4>, rec_warp_bytes<R, COMP, 32>(0));
            } else {
                if (tile_c == 8)
                    launch_recs(k_grid_tiles_recs<R, COMP, KM_SEP, 8, 4>, rec_warp_bytes<R, COMP, 8>(sep_len));
                else if (tile_c == 16)
                    launch_recs(k_grid_tiles_recs<R, COMP, KM_SEP, 16, 4>, rec_warp_bytes<R, COMP, 16>(sep_len));
                else
                    launch_recs(k_grid_tiles_recs<R, COMP, KM_SEP, 32, 4>, rec_warp_bytes<R, COMP, 32>(sep_len));
            }
        } else if (use_cols && kind == GK_WPROJ)
            b ? (t32 ? launch(k_grid_tiles<R, COMP, KM_WPROJ, true, 32, 1>) : launch(k_grid_tiles<R, COMP, KM_WPROJ, true, 16, 1>))
              : (t32 ? launch(k_grid_tiles<R, COMP, KM_WPROJ, false, 32, 1>) : launch(k_grid_tiles<R, COMP, KM_WPROJ, false, 16, 1>));
        else if (use_cols)
            b ? (t32 ? launch(k_grid_tiles<R, COMP, KM_SEP, true, 32, 1>) : launch(k_grid_tiles<R, COMP, KM_SEP, true, 16, 1>))
              : (t32 ? launch(k_grid_tiles<R, COMP, KM_SEP, false, 32, 1>) : launch(k_grid_tiles<R, COMP, KM_SEP, false, 16, 1>));
        else if (use_taps && tile_c == 8) {
            // four 8-column tiles per block (k_grid_tiles_mw)
            const int tb = int((smem + 15) / 16 * 16);
            auto launch_mw = [&](auto kern) {
                const size_t bs = size_t(4) * size_t(tb);
                if (bs > 48 * 1024)
                    STPGPU_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bs)));
                c->mark(1);
                kern<<<unsigned((ntiles + 3) / 4), 128, bs, st>>>(gp, ntiles, tb);
                STPGPU_CHECK_LAUNCH();
                c->mark(2);
            };
            if (kind == GK_WPROJ)
                b ? launch_mw(k_grid_tiles_mw<R, COMP, KM_WPROJ, true, 8, 4>)
                  : launch_mw(k_grid_tiles_mw<R, COMP, KM_WPROJ, false, 8, 4>);
            else
                b ? launch_mw(k_grid_tiles_mw<R, COMP, KM_SEP, true, 8, 4>)
                  : launch_mw(k_grid_tiles_mw<R, COMP, KM_SEP, false, 8, 4>);
        } else if (use_taps && kind == GK_WPROJ)
            b ? (t32 ? launch(k_grid_tiles<R, COMP, KM_WPROJ, true, 32, 2>) : launch(k_grid_tiles<R, COMP, KM_WPROJ, true, 16, 2>))
              : (t32 ? launch(k_grid_tiles<R, COMP, KM_WPROJ, false, 32, 2>) : launch(k_grid_tiles<R, COMP, KM_WPROJ, false, 16, 2>));
        else if (use_taps)
            b ? (t32 ? launch(k_grid_tiles<R, COMP, KM_SEP, true, 32, 2>) : launch(k_grid_tiles<R, COMP, KM_SEP, true, 16, 2>))
              : (t32 ? launch(k_grid_tiles<R, COMP, KM_SEP, false, 32, 2>) : launch(k_grid_tiles<R, COMP, KM_SEP, false, 16, 2>));
        else if (kind == GK_WPROJ)
            b ? (t32 ? launch(k_grid_tiles<R, COMP, KM_WPROJ, true, 32>) : launch(k_grid_tiles<R, COMP, KM_WPROJ, true, 16>))
              : (t32 ? launch(k_grid_tiles<R, COMP, KM_WPROJ, false, 32>) : launch(k_grid_tiles<R, COMP, KM_WPROJ, false, 16>));
        else if (kind == GK_EXACT)
            b ? (t32 ? launch(k_grid_tiles<R, COMP, KM_EXACT, true, 32>) : launch(k_grid_tiles<R, COMP, KM_EXACT, true, 16>))
              : (t32 ? launch(k_grid_tiles<R, COMP, KM_EXACT, false, 32>) : launch(k_grid_tiles<R, COMP, KM_EXACT, false, 16>));
        else
            b ? (t32 ? launch(k_grid_tiles<R, COMP, KM_SEP, true, 32>) : launch(k_grid_tiles<R, COMP, KM_SEP, true, 16>))
              : (t32 ? launch(k_grid_tiles<R, COMP, KM_SEP, false, 32>) : launch(k_grid_tiles<R, COMP, KM_SEP, false, 16>));
    } else {
        c->mark(1);
        c->mark(2);
    }
    g.grid = grid;
    g.beam = beam;
    return g;
}

struct ScalarsBack {
    double total;
    unsigned long long ngood;
    uint32_t nitems;
    unsigned int err;
    int max_support;
};

ScalarsBack read_back(stpgpu_context* c, const GridOut& g)
{
    // the scalars packed by one kernel straight into the page-locked stage
    ScalarPack* h = c->host_stage<ScalarPack>(1);
    k_pack_scalars<<<1, 32, 0, c->stream>>>(g.d_total, g.d_ngood, g.d_nitems, g.d_err, g.d_plane_support,
        g.nplanes > 0 ? g.nplanes : 0, c->host_stage_dev(h));
    STPGPU_CHECK_LAUNCH();
    STPGPU_CUDA_TRY(cudaStreamSynchronize(c->stream));
    ScalarsBack r { h->total, h->ngood, h->nitems, h->err, h->max_support };
    // bit 4: the 32-bit |w| sort met a long run of distinct |w| (the caller
    // repeats the gridding with the 64-bit sort); bit 8: the staged
    // gridder's records exceeded their capacity (the caller grids again with
    // the buffer sized from the count); bit 16: the W-planes without the
    // sort did not apply (the caller grids again on the sorting path); other
    // bits are errors
    if (r.err & ~(4u | 8u | 16u))
        fail(STPGPU_ERR_DEVICE, "gridder reported internal error flags " + std::to_string(r.err));
    return r;
}

template <typename R>
const double* device_gcf(stpgpu_context* c, const ImagerSetup& s)
{
    double* gcf = c->buf<double>("gcf", s.N);
    c->buf<double>("gcfinv", s.N);
    if (c->memo("gcf", std::to_string(s.kf) + "/" + fkey(s.trunc) + "/" + std::to_string(s.N) + "/"
                          + std::to_string(s.analytic))
        && c->memo("gcfinv", std::to_string(s.kf) + "/" + fkey(s.trunc) + "/" + std::to_string(s.N) + "/"
            + std::to_string(s.analytic)))
        return gcf;
    c->memo("gcfinv", std::to_string(s.kf) + "/" + fkey(s.trunc) + "/" + std::to_string(s.N) + "/"
            + std::to_string(s.analytic));
    double ksum_inv = 1.0;
    const int dmax = int(std::floor(s.trunc)) + 1;
    if (!s.analytic) {
        const int centre = s.N / 2;
        double ssum = 0.0;
        for (int d = -std::min(dmax, centre); d <= std::min(dmax, s.N - centre - 1); d++)
            ssum += kernel_value(s.kf, s.trunc, double(d));
        ksum_inv = ssum > 0.0 ? 1.0 / ssum : 1.0;
    }
    k_imgdom_kernel<<<grid1d(s.N, 256), 256, 0, c->stream>>>(s.kf, s.trunc, s.N, s.analytic, ksum_inv, dmax, gcf);
    STPGPU_CHECK_LAUNCH();
    double* ginv = c->buf<double>("gcfinv", s.N);
    k_reciprocal<<<grid1d(s.N, 256), 256, 0, c->stream>>>(gcf, ginv, s.N);
    STPGPU_CHECK_LAUNCH();
    return gcf;
}

// c2r FFT + crop/normalise of a gridded snapshot (fft.cpp:45-135,
// imager.h:97-213) on the context's current stream.
template <typename R>
void finish_imager(stpgpu_context* c, const ImagerSetup& s, int image_size, int correction, const GridOut& g,
    void* d_image, void* d_beam, int out_f32)
{
    if constexpr (sizeof(R) == 4) {
        if (s.wide_fft) { // the gridder wrote double2 cells: Z2D + double normalisation
            finish_imager<double>(c, s, image_size, correction, g, d_image, d_beam, out_f32);
            return;
        }
    }
    cudaStream_t st = c->stream;
    const int N = s.N;
    R* img = c->buf<R>("fftimg", size_t(N) * N);
    const cufftType type = sizeof(R) == 8 ? CUFFT_Z2D : CUFFT_C2R;
    cufftHandle h = c->plan(N, type);
    auto exec = [&](void* in, R* out) {
        cufftResult r;
        if (sizeof(R) == 8)
            r = cufftExecZ2D(h, reinterpret_cast<cufftDoubleComplex*>(in), reinterpret_cast<cufftDoubleReal*>(out));
        else
            r = cufftExecC2R(h, reinterpret_cast<cufftComplex*>(in), reinterpret_cast<cufftReal*>(out));
        if (r != CUFFT_SUCCESS)
            fail(STPGPU_ERR_CUFFT, "cuFFT c2r execution failed (" + std::to_string(int(r)) + ")");
    };
    const double* gcf = correction ? device_gcf<R>(c, s) : nullptr;
    const double* ginv = correction ? c->buf<double>("gcfinv", s.N) : nullptr;
    (void)gcf;
    const dim3 ngrid(std::min<unsigned>(grid1d(image_size, 256), 4), image_size);
    // 16-byte path: every 4-row group inside one crop segment and aligned
    const bool vec4 = (image_size % 8) == 0 && (N % 4) == 0
        && (reinterpret_cast<uintptr_t>(d_image) % 16) == 0 && (!d_beam || (reinterpret_cast<uintptr_t>(d_beam) % 16) == 0);
    const dim3 ngrid4(grid1d(image_size / 4, 256), (image_size + kNormCols - 1) / kNormCols);
    auto normalise = [&](void* out) {
        if (vec4) {
            if (out_f32)
                k_normalise4<R, float><<<ngrid4, 256, 0, st>>>(img, N, image_size, g.d_total, ginv, correction,
                    reinterpret_cast<float*>(out));
            else
                k_normalise4<R, double><<<ngrid4, 256, 0, st>>>(img, N, image_size, g.d_total, ginv, correction,
                    reinterpret_cast<double*>(out));
            STPGPU_CHECK_LAUNCH();
            return;
        }
        if (out_f32)
            k_normalise<R, float><<<ngrid, 256, 0, st>>>(img, N, image_size, g.d_total, ginv, correction,
                reinterpret_cast<float*>(out));
        else
            k_normalise<R, double><<<ngrid, 256, 0, st>>>(img, N, image_size, g.d_total, ginv, correction,
                reinterpret_cast<double*>(out));
        STPGPU_CHECK_LAUNCH();
    };
    exec(g.grid, img);
    c->mark(3);
    normalise(d_image);
    c->mark(4);
    if (s.beam && d_beam) {
        exec(g.beam, img);
        normalise(d_beam);
    }
}

// Compensated FP32 keeps the grid in double and runs the c2r in double
// precision when the grid correction would amplify the single-precision
// transform's rounding past the 1e-5 peak-relative bound.  Normalisation
// divides pixel (i, j) by gcf[i] gcf[j] (imager.h:97-150), so an error that
// the FP32 c2r leaves at about 4e-10 of the peak (measured on an 8192^2
// PSWF image with analytic correction: 2.3e-5 of the peak at
// 1/gcf_min^2 = 6.2e4, against 2.2e-6 for an FP32 grid transformed in
// double) is multiplied by up to 1/gcf_min^2 over the output field.  Rule:
// wide when 1/gcf_min^2 > 4096, i.e. an expected FP32-c2r error above about
// 1.5e-6 of the peak.  GaussianSinc S=3 with the DFT correction (1/gcf_min^2
// = 890) keeps the FP32 transform; PSWF (1.5e4 with the DFT correction at
// S=3, 6.2e4 analytic) takes the wide one.  The gcf values are those of
// k_imgdom_kernel (ImgDomKernel, conv_func.h:351-412) over the kept field.
constexpr double kWideFftAmplification = 4096.0;

bool wide_fft_rule(const ImagerSetup& s, int image_size, int correction)
{
    if (!correction)
        return false;
    const int N = s.N, centre = N / 2, hs = image_size / 2;
    double gmin = 1e300;
    if (s.analytic) {
        for (int m = -hs; m < hs; m++)
            gmin = std::min(gmin, std::fabs(gcf_value(s.kf, double(m) / centre)));
    } else {
        const int dmax = int(std::floor(s.trunc)) + 1;
        const int dlo = -std::min(dmax, centre), dhi = std::min(dmax, N - centre - 1);
        double ssum = 0.0;
        for (int d = dlo; d <= dhi; d++)
            ssum += kernel_value(s.kf, s.trunc, double(d));
        const double kinv = ssum > 0.0 ? 1.0 / ssum : 1.0;
        for (int m = 0; m <= hs; m++) {
            double r = 0.0;
            for (int d = dlo; d <= dhi; d++) {
                const long long jm = (long long)(d < 0 ? d + N : d) * m % N;
                r += kernel_value(s.kf, s.trunc, double(d)) * kinv * std::cos(2.0 * M_PI * double(jm) / double(N));
            }
            gmin = std::min(gmin, std::fabs(r));
        }
    }
    return !(gmin > 0.0) || 1.0 / (gmin * gmin) > kWideFftAmplification;
}

// wide_fft_rule memoised for the process (the DFT form costs a few thousand
// cosines per evaluation); used by the imaging calls and the server's
// admission estimate
bool wide_fft_needed(const ImagerSetup& s, int image_size, int correction)
{
    static std::mutex mu;
    static std::map<std::string, bool> memo;
    const std::string key = std::to_string(s.kf) + "/" + fkey(s.trunc) + "/" + std::to_string(s.N) + "/"
        + std::to_string(s.analytic) + "/" + std::to_string(image_size) + "/" + std::to_string(correction);
    std::lock_guard<std::mutex> lock(mu);
    auto it = memo.find(key);
    if (it != memo.end())
        return it->second;
    const bool wide = wide_fft_rule(s, image_size, correction);
    memo[key] = wide;
    return wide;
}

// stp::image_visibilities (imager.h:233-376) on device buffers.  The whole
// pipeline is enqueued without a host round trip; the normalisation reads
// the sampling total on the device, and the scalars are read back once at
// the end (an empty result, imager.h:355, is reported then).
template <typename R, int COMP>
void run_imager(stpgpu_context* c, const ImagerSetup& s_in, int image_size, int correction, const void* d_vis,
    int vis_c64, const double* d_wts, const double* d_uvw, int64_t n, void* d_image, void* d_beam, int out_f32,
    stpgpu_imager_info* info, bool graphable = false)
{
    if (image_size <= 0 || image_size > s_in.N || (image_size % 2) != 0)
        fail(STPGPU_ERR_INVALID_ARG, "image_size must be even, > 0 and <= padded_image_size");
    ImagerSetup s = s_in;
    s.wide_fft = (COMP == 1 && wide_fft_needed(s, image_size, correction)) ? 1 : 0;
    // W-planes without the |w| sort where they apply (mean |w| per plane, no
    // A-projection time steps); a size class whose data did not allow it on
    // its last call (visibilities outside the grid, non-finite w) sorts
    s.wsel = s.nplanes > 0 && s.nplanes <= WSEL_MAXP && !s.wmedian && s.ntimesteps == 0 && !s.full_wsort
        && n < (int64_t(1) << 31);
    // tile width: the autotuned choice of this size class; the first call of
    // a class grids with both widths, times them, keeps the faster for later
    // calls (every pass produces the complete grid; the last one is used)
    const int precision = sizeof(R) == 8 ? STPGPU_FP64 : (COMP ? STPGPU_FP32C : STPGPU_FP32);
    const std::string cls = size_class(s, precision);
    if (s.wsel && c->wsel_off.count(cls))
        s.wsel = 0;
    GridOut g;
    // STPGPU_GRIDDER_LAYOUT=32|16|32c|16c|32t|16t|8t|32r|16r|8r pins the tile
    // width and gridder form (c: column-packed, t: lane-per-tap, r: staged
    // records) instead of the autotuner's choice
    if (const char* pin = std::getenv("STPGPU_GRIDDER_LAYOUT")) {
        const int w = std::atoi(pin);
        if (w == 16 || w == 32 || (w == 8 && (std::strchr(pin, 't') || std::strchr(pin, 'r'))))
            c->tune_set(cls,
                w | (std::strchr(pin, 'c') ? kLayoutCols : 0) | (std::strchr(pin, 't') ? kLayoutTaps : 0)
                    | (std::strchr(pin, 'r') ? kLayoutRecs : 0));
    }
    int tuned_lay = 0;
    const bool have_tune = c->tune_get(cls, tuned_lay);
    // Device-pointer calls that repeat the previous call exactly (parameters,
    // sizes, buffers) replay a CUDA graph of the gridding, FFT and
    // normalisation kernels, captured on the first repeat; any other call
    // drops it.  The data in the buffers may change between calls.
    std::string sig;
    if (graphable && !c->timing && !large_support(s) && s.ntimesteps == 0) {
        auto put = [&](const void* q, size_t nb) { sig.append(reinterpret_cast<const char*>(q), nb); };
        put(&precision, sizeof(precision));
        put(&s, sizeof(s));
        put(&image_size, sizeof(image_size));
        put(&correction, sizeof(correction));
        put(&vis_c64, sizeof(vis_c64));
        put(&n, sizeof(n));
        put(&out_f32, sizeof(out_f32));
        const void* ptrs[6] = { d_vis, d_wts, d_uvw, d_image, d_beam, reinterpret_cast<const void*>(c->stream) };
        put(ptrs, sizeof(ptrs));
    }
    const bool repeat = !sig.empty() && sig == c->single_sig;
    if (!repeat)
        c->drop_single();
    if (repeat && c->single_exec) {
        STPGPU_CUDA_TRY(cudaGraphLaunch(c->single_exec, c->stream));
        g_launches += c->single_launches; // the replay runs the captured kernels
        g = c->single_g;
    } else if (repeat && have_tune) {
        const int before = g_launches;
        STPGPU_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        try {
            g = run_gridder<R, COMP>(c, s, d_vis, vis_c64, d_wts, d_uvw, 0, n, tuned_lay & 0xff, nullptr,
                form_of(tuned_lay));
            finish_imager<R>(c, s, image_size, correction, g, d_image, d_beam, out_f32);
        } catch (...) {
            cudaGraph_t dead = nullptr;
            cudaStreamEndCapture(c->stream, &dead);
            if (dead)
                cudaGraphDestroy(dead);
            c->drop_single();
            throw;
        }
        STPGPU_CUDA_TRY(cudaStreamEndCapture(c->stream, &c->single_graph));
        int zk = 0;
        c->single_graph = memsets_to_kernels(c->single_graph, &zk);
        g_launches += zk;
        STPGPU_CUDA_TRY(cudaGraphInstantiate(&c->single_exec, c->single_graph, 0));
        STPGPU_CUDA_TRY(cudaGraphLaunch(c->single_exec, c->stream));
        c->single_g = g;
        c->single_launches = g_launches - before;
    } else if (have_tune || c->timing) {
        const int lay = have_tune ? tuned_lay : TILE_C_DEFAULT;
        g = run_gridder<R, COMP>(c, s, d_vis, vis_c64, d_wts, d_uvw, 0, n, lay & 0xff, nullptr,
            form_of(lay));
    } else {
        for (auto& e : c->tev)
            if (!e)
                STPGPU_CUDA_TRY(cudaEventCreate(&e));
        // an untimed pass first grows every buffer (16 columns: the most
        // tiles) and fills the cached tables, so no timed pass pays that
        // the column-packed form is a candidate for large kernels only (with
        // K <= 17 the lane-per-item form is faster on every measured workload)
        g = run_gridder<R, COMP>(c, s, d_vis, vis_c64, d_wts, d_uvw, 0, n, 16);
        // the widest kernel the data actually uses (W-planes are truncated
        // below the maximum support), read back from the untimed pass
        const int used_support = s.nplanes > 0 ? std::max(read_back(c, g).max_support, 0) : s.support;
        // the clipped forms need one footprint segment per axis and tile
        const bool clip_ok = !s.kernel_exact && s.N >= 2 * (2 * (s.nplanes > 0 ? s.max_support : s.support) + 33) + 2;
        std::vector<int> lays = { 32, 16 };
        if (clip_ok) {
            for (int w : { 32 | kLayoutTaps, 16 | kLayoutTaps, 8 | kLayoutTaps })
                lays.push_back(w);
            if (2 * used_support + 1 > 17)
                for (int w : { 32 | kLayoutCols, 16 | kLayoutCols })
                    lays.push_back(w);
            if (!s.beam)
                for (int w : { 32 | kLayoutRecs, 16 | kLayoutRecs, 8 | kLayoutRecs })
                    lays.push_back(w);
        }
        const int ncand = int(lays.size());
        std::vector<float> ms(size_t(ncand), 1e30f);
        // each candidate timed twice, the faster pass kept (single passes
        // of close candidates swap order from run to run)
        for (int rep = 0; rep < 2; rep++)
            for (int k = 0; k < ncand; k++) {
                STPGPU_CUDA_TRY(cudaEventRecord(c->tev[0], c->stream));
                g = run_gridder<R, COMP>(c, s, d_vis, vis_c64, d_wts, d_uvw, 0, n, lays[k] & 0xff, nullptr,
                    form_of(lays[k]));
                STPGPU_CUDA_TRY(cudaEventRecord(c->tev[1], c->stream));
                STPGPU_CUDA_TRY(cudaEventSynchronize(c->tev[1]));
                float t = 0.f;
                STPGPU_CUDA_TRY(cudaEventElapsedTime(&t, c->tev[0], c->tev[1]));
                ms[k] = std::min(ms[k], t);
            }
        int best = 0;
        for (int k = 1; k < ncand; k++)
            if (ms[k] < ms[best])
                best = k;
        c->tune_set(cls, lays[best]);
        if (std::getenv("STPGPU_LOG_TUNING")) {
            std::string line;
            for (int k = 0; k < ncand; k++) {
                const int f = form_of(lays[k]);
                line += " " + std::to_string(lays[k] & 0xff)
                    + (f == 1 ? "c" : (f == 2 ? "t" : (f == 3 ? "r" : ""))) + " " + std::to_string(ms[k]);
            }
            std::fprintf(stderr, "stpgpu gridder tuner: %s (layout ms):%s -> candidate %d (single call)\n", cls.c_str(),
                line.c_str(), best);
        }
    }
    if (!(repeat && c->single_exec))
        finish_imager<R>(c, s, image_size, correction, g, d_image, d_beam, out_f32);
    if (!sig.empty())
        c->single_sig = sig;
    const int N = s.N;
    ScalarsBack sb = read_back(c, g);
    if (sb.err & 8u) {
        // records outgrew the remembered capacity: size them from a fresh
        // count (the next run_gridder reads the total) and grid again
        for (auto it = c->rec_ratio.begin(); it != c->rec_ratio.end();)
            it = it->first.compare(0, c->ns.size() + 1, c->ns + "/") == 0 ? c->rec_ratio.erase(it) : std::next(it);
        c->drop_single();
        int lay = TILE_C_DEFAULT;
        c->tune_get(cls, lay);
        g = run_gridder<R, COMP>(c, s, d_vis, vis_c64, d_wts, d_uvw, 0, n, lay & 0xff, nullptr, form_of(lay));
        finish_imager<R>(c, s, image_size, correction, g, d_image, d_beam, out_f32);
        sb = read_back(c, g);
    }
    if (sb.err & 16u) {
        // the W-planes without the sort did not apply: the sorting path, for
        // this call and the size class's next ones
        c->wsel_off.insert(cls);
        c->drop_single();
        s.wsel = 0;
        int lay = TILE_C_DEFAULT;
        c->tune_get(cls, lay);
        g = run_gridder<R, COMP>(c, s, d_vis, vis_c64, d_wts, d_uvw, 0, n, lay & 0xff, nullptr, form_of(lay));
        finish_imager<R>(c, s, image_size, correction, g, d_image, d_beam, out_f32);
        sb = read_back(c, g);
    }
    if ((sb.err & 4u) && !s.full_wsort) {
        // rare data (many distinct |w| within one single-precision step): redo with the 64-bit |w| sort
        ImagerSetup s64 = s;
        s64.full_wsort = 1;
        int lay = TILE_C_DEFAULT;
        c->tune_get(cls, lay);
        g = run_gridder<R, COMP>(c, s64, d_vis, vis_c64, d_wts, d_uvw, 0, n, lay & 0xff, nullptr,
            form_of(lay));
        finish_imager<R>(c, s64, image_size, correction, g, d_image, d_beam, out_f32);
        sb = read_back(c, g);
    }
    if (info) {
        info->sample_grid_total = sb.total;
        info->n_good_vis = int64_t(sb.ngood);
        info->n_grid_items = sb.nitems;
        info->padded_image_size = N;
        info->num_wplanes = s.nplanes;
        info->max_plane_support = sb.max_support;
        info->flags = s.wide_fft ? 1 : 0;
        info->image_size = sb.total > 0.0 ? image_size : 0;
        if (c->timing) {
            float ms[4] = { 0, 0, 0, 0 };
            for (int k = 0; k < 4; k++)
                STPGPU_CUDA_TRY(cudaEventElapsedTime(&ms[k], c->pev[k], c->pev[k + 1]));
            for (int k = 0; k < 4; k++)
                info->phase_ms[k] = ms[k];
        }
    }
}

ImagerSetup setup_from(const stpgpu_imager_pars* p, const stpgpu_wproj_pars* w, const stpgpu_aproj_pars* a,
    int& image_size)
{
    if (!p)
        fail(STPGPU_ERR_INVALID_ARG, "null imager parameters");
    if (p->kernel_function < 0 || p->kernel_function > 5)
        fail(STPGPU_ERR_INVALID_ARG, "unknown kernel function");
    if (!(p->cell_size > 0.0))
        fail(STPGPU_ERR_INVALID_ARG, "cell_size must be > 0");
    if (!(p->padding_factor >= 1.0))
        fail(STPGPU_ERR_INVALID_ARG, "padding_factor must be >= 1");
    ImagerSetup s;
    image_size = p->image_size;
    s.N = p->padded_image_size > 0 ? p->padded_image_size : int(unsigned(double(image_size) * p->padding_factor));
    s.kf = p->kernel_function;
    s.support = p->kernel_support;
    s.trunc = double(p->kernel_support);
    s.kernel_exact = p->kernel_exact;
    s.os = p->oversampling;
    s.beam = p->generate_beam;
    s.analytic = p->analytic_gcf;
    s.cell_size = p->cell_size;
    s.shift_uv = 1;
    s.halfplane = 1;
    if (w && w->num_wplanes > 0) {
        if (p->kernel_exact)
            fail(STPGPU_ERR_INVALID_ARG, "W-projection cannot be used with kernel_exact (imager.h:287)");
        s.nplanes = w->num_wplanes;
        s.max_support = w->max_wpconv_support;
        s.undersampling = w->undersampling_opt;
        s.trunc_perc = w->kernel_trunc_perc;
        s.wmedian = w->wplanes_median;
        if (w->hankel_opt) {
            // InterpType (types.h:55-59): LINEAR 0, CUBIC 1, COSINE 2 (interpolated linearly,
            // aw_projection.cpp:263-266)
            if (w->interp_type < 0 || w->interp_type > 2)
                fail(STPGPU_ERR_INVALID_ARG, "unknown interp_type");
            s.hankel = 1;
            s.proj_slice = w->hankel_proj_slice ? 1 : 0;
            s.cubic = w->interp_type == 1;
        }
    }
    if (!p->kernel_exact && p->oversampling < 1)
        fail(STPGPU_ERR_INVALID_ARG, "oversampling must be >= 1 when kernel_exact is false");
    if (a && a->num_timesteps > 0) {
        // imager.h:274-283
        if (s.nplanes <= 0)
            fail(STPGPU_ERR_INVALID_ARG, "W-projection must be used when A-projection is enabled.");
        if (s.hankel)
            fail(STPGPU_ERR_INVALID_ARG, "Hankel transform cannot be used when A-projection is enabled.");
        if (a->num_timesteps > 255 || int64_t(a->num_timesteps) * s.nplanes > 65535)
            fail(STPGPU_ERR_UNSUPPORTED, "A-projection supports at most 255 time steps and 65535 planes x steps");
        if (a->n_pbeam_coefs < 1 || !a->pbeam_coefs)
            fail(STPGPU_ERR_INVALID_ARG, "A-projection needs the primary beam coefficients");
        s.ntimesteps = a->num_timesteps;
        s.aproj_opt = a->aproj_opt ? 1 : 0;
        s.obs_dec = (a->obs_dec * M_PI) / 180.0; // deg2rad, global_macros.h:40
        s.obs_ra = (a->obs_ra * M_PI) / 180.0;
        s.lha = a->lha;
        s.pbcoefs = a->pbeam_coefs;
        s.npbcoefs = a->n_pbeam_coefs;
    }
    return s;
}

template <typename T>
T* to_device(stpgpu_context* c, const char* name, const void* host, size_t count)
{
    T* d = c->buf<T>(name, count);
    if (count)
        STPGPU_CUDA_TRY(cudaMemcpyAsync(d, host, sizeof(T) * count, cudaMemcpyHostToDevice, c->stream));
    return d;
}

// ------------------------------------------------------------------ batch

constexpr int kBatchStreams = 8;

struct BatchSnap {
    ImagerSetup s;
    int image_size = 0;
    int correction = 1;
    const void* vis = nullptr; // caller's pointers (device or host)
    int c64 = 0;
    const double* wts = nullptr;
    const double* uvw = nullptr;
    int64_t n = 0;
    void* image = nullptr;
    std::string cls; // size class of the tile autotuner
    int tile_c = TILE_C_DEFAULT;
    int persist = 0;
    int form = 0; // gridder form: 0 lanes-per-item, 2 lane-per-tap
};

// Tuned layout of a batch snapshot.  The lane-per-tap form clips footprints
// to tiles and needs one segment per axis and tile (as in run_gridder).
void apply_layout(BatchSnap& b, int lay)
{
    b.tile_c = lay & 0xff;
    b.persist = (lay & kLayoutPersist) ? 1 : 0;
    const int conv = b.s.nplanes > 0 ? b.s.max_support : b.s.support;
    const bool clip_ok = !b.s.kernel_exact && b.s.N >= 2 * (2 * conv + 1 + 32) + 2;
    // the staged form: run_gridder falls back to the lane-per-tap form where
    // it does not apply and reports the form it built in GridLaunch::form
    b.form = ((lay & kLayoutRecs) && clip_ok) ? 3 : (((lay & kLayoutTaps) && clip_ok) ? 2 : 0);
}

void batch_streams(stpgpu_context* c)
{
    if (!c->wstreams.empty())
        return;
    for (int k = 0; k < kBatchStreams; k++) {
        cudaStream_t w;
        STPGPU_CUDA_TRY(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking));
        c->wstreams.push_back(w);
        cudaEvent_t e;
        STPGPU_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->wevents.push_back(e);
    }
    STPGPU_CUDA_TRY(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
}

// main stream -> every worker stream
void batch_fork(stpgpu_context* c, cudaStream_t main)
{
    STPGPU_CUDA_TRY(cudaEventRecord(c->fork_ev, main));
    for (auto w : c->wstreams)
        STPGPU_CUDA_TRY(cudaStreamWaitEvent(w, c->fork_ev, 0));
}

// every worker stream -> main stream
void batch_join(stpgpu_context* c, cudaStream_t main)
{
    for (size_t k = 0; k < c->wstreams.size(); k++) {
        STPGPU_CUDA_TRY(cudaEventRecord(c->wevents[k], c->wstreams[k]));
        STPGPU_CUDA_TRY(cudaStreamWaitEvent(main, c->wevents[k], 0));
    }
}

template <typename R, int COMP, int KMODE, int TC, bool PERSIST, int FORM>
void launch_grid_batch(cudaStream_t st, size_t smem, const BatchGridParams<R>& P, uint32_t total_tiles, bool capturing)
{
    auto kern = k_grid_batch<R, COMP, KMODE, false, TC, PERSIST, FORM>;
    if (!capturing && smem > 48 * 1024)
        STPGPU_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    uint32_t blocks = std::max<uint32_t>(1, total_tiles);
    if (PERSIST) {
        static int sms = 0;
        if (sms == 0) {
            int dev = 0;
            STPGPU_CUDA_TRY(cudaGetDevice(&dev));
            STPGPU_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        }
        int per_sm = 0;
        STPGPU_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32, smem));
        blocks = std::min<uint32_t>(blocks, uint32_t(std::max(per_sm, 1) * sms));
    }
    kern<<<blocks, 32, smem, st>>>(P);
    STPGPU_CHECK_LAUNCH();
}


template <typename R, int COMP, int KMODE, int FORM>
void launch_mode_form(cudaStream_t st, int layout, size_t smem, const BatchGridParams<R>& P, uint32_t total, bool cap)
{
    const bool t32 = (layout & 0xff) == 32;
    if (layout & kLayoutPersist)
        t32 ? launch_grid_batch<R, COMP, KMODE, 32, true, FORM>(st, smem, P, total, cap)
            : launch_grid_batch<R, COMP, KMODE, 16, true, FORM>(st, smem, P, total, cap);
    else
        t32 ? launch_grid_batch<R, COMP, KMODE, 32, false, FORM>(st, smem, P, total, cap)
            : launch_grid_batch<R, COMP, KMODE, 16, false, FORM>(st, smem, P, total, cap);
}

template <typename R, int COMP, int KMODE>
void launch_mode(cudaStream_t st, int layout, size_t smem, const BatchGridParams<R>& P, uint32_t total, bool cap)
{
    if (KMODE != KM_EXACT && (layout & kLayoutRecs))
        launch_mode_form<R, COMP, KMODE, 3>(st, layout, smem, P, total, cap);
    else if (KMODE != KM_EXACT && (layout & kLayoutTaps))
        launch_mode_form<R, COMP, KMODE, 2>(st, layout, smem, P, total, cap);
    else
        launch_mode_form<R, COMP, KMODE, 0>(st, layout, smem, P, total, cap);
}

template <typename R, int COMP>
void launch_group(cudaStream_t st, int kind, int layout, size_t smem, const BatchGridParams<R>& P, uint32_t total,
    bool capturing)
{
    if (kind == GK_WPROJ)
        launch_mode<R, COMP, KM_WPROJ>(st, layout, smem, P, total, capturing);
    else if (kind == GK_EXACT)
        launch_mode<R, COMP, KM_EXACT>(st, layout, smem, P, total, capturing);
    else
        launch_mode<R, COMP, KM_SEP>(st, layout, smem, P, total, capturing);
}

// Enqueue one batch: preparation of every snapshot on the worker streams,
// persistent gridder launches on the main stream (one per kernel variant,
// or one per size class when class_ms is given, each timed), then c2r +
// normalisation per snapshot on the worker streams, and the scalars of every
// snapshot gathered into `scal` (pinned host memory) by the main stream.
template <typename R, int COMP>
int batch_enqueue(stpgpu_context* c, std::vector<BatchSnap>& B, int out_f32, int device_ptrs, bool capturing,
    BatchScalars* scal, unsigned char* host_params, std::map<std::string, float>* class_ms)
{
    const cudaStream_t main = c->stream;
    const int nb = int(B.size());
    const int K = int(c->wstreams.size());
    const size_t vb = 16;
    std::vector<GridLaunch<R>> L(nb);
    std::vector<GridOut> G(nb);
    std::vector<void*> dimg(nb);
    if (!device_ptrs && !class_ms) {
        // host buffers: each snapshot runs its whole pipeline on its worker
        // stream (H2D, preparation, gridder, c2r, normalisation, D2H), so the
        // transfers of one snapshot overlap the compute of the others
        batch_fork(c, main);
        for (int i = 0; i < nb; i++) {
            c->stream = c->wstreams[i % K];
            c->ns = "b" + std::to_string(i) + "/";
            BatchSnap& b = B[i];
            const void* dv = to_device<unsigned char>(c, "in_vis", b.vis, (b.c64 ? 8 : vb) * size_t(b.n));
            const double* dw = to_device<double>(c, "in_w", b.wts, size_t(b.n));
            const double* duvw = to_device<double>(c, "in_uvw", b.uvw, 3 * size_t(b.n));
            const size_t ob = (out_f32 ? 4 : 8) * size_t(b.image_size) * b.image_size;
            void* di = c->buf<unsigned char>("out_img", ob);
            GridOut g = run_gridder<R, COMP>(c, b.s, dv, b.c64, dw, duvw, 0, b.n, b.tile_c, nullptr, b.form);
            finish_imager<R>(c, b.s, b.image_size, b.correction, g, di, nullptr, out_f32);
            BatchScalars* ds = c->buf<BatchScalars>("scal", 1);
            k_collect_scalars<<<1, 1, 0, c->stream>>>(g.d_total, g.d_ngood, g.d_nitems, g.d_err,
                g.d_plane_support ? g.d_plane_support : reinterpret_cast<const int*>(g.d_err),
                g.d_plane_support ? g.nplanes : 0, ds);
            STPGPU_CHECK_LAUNCH();
            STPGPU_CUDA_TRY(cudaMemcpyAsync(&scal[i], ds, sizeof(BatchScalars), cudaMemcpyDeviceToHost, c->stream));
            STPGPU_CUDA_TRY(cudaMemcpyAsync(b.image, di, ob, cudaMemcpyDeviceToHost, c->stream));
        }
        c->stream = main;
        c->ns = "";
        batch_join(c, main);
        return nb;
    }
    batch_fork(c, main);
    for (int i = 0; i < nb; i++) {
        c->stream = c->wstreams[i % K];
        c->ns = "b" + std::to_string(i) + "/";
        BatchSnap& b = B[i];
        const void* dv = b.vis;
        const double* dw = b.wts;
        const double* duvw = b.uvw;
        dimg[i] = b.image;
        if (!device_ptrs) {
            const size_t vbytes = b.c64 ? 8 : vb;
            dv = to_device<unsigned char>(c, "in_vis", b.vis, vbytes * size_t(b.n));
            dw = to_device<double>(c, "in_w", b.wts, size_t(b.n));
            duvw = to_device<double>(c, "in_uvw", b.uvw, 3 * size_t(b.n));
            dimg[i] = c->buf<unsigned char>("out_img", (out_f32 ? 4 : 8) * size_t(b.image_size) * b.image_size);
        }
        G[i] = run_gridder<R, COMP>(c, b.s, dv, b.c64, dw, duvw, 0, b.n, b.tile_c, &L[i], b.form);
    }
    c->stream = main;
    c->ns = "batch/";
    batch_join(c, main);

    // ---- persistent gridder launches over (snapshot, tile) work queues
    std::map<std::string, std::vector<int>> groups;
    for (int i = 0; i < nb; i++) {
        if (L[i].kind == GK_NONE || L[i].ntiles == 0)
            continue;
        std::string key = std::to_string(L[i].kind) + "/" + std::to_string(L[i].tile_c) + "/"
            + std::to_string(B[i].persist) + "/" + std::to_string(L[i].form);
        if (class_ms)
            key += "|" + B[i].cls;
        groups[key].push_back(i);
    }
    int gi = 0, nlaunch = 0;
    for (auto& kv : groups) {
        const std::vector<int>& all = kv.second;
        for (size_t c0 = 0; c0 < all.size(); c0 += kBatchGrid) {
            const int m = int(std::min<size_t>(kBatchGrid, all.size() - c0));
            auto* P = reinterpret_cast<BatchGridParams<R>*>(host_params); // host-side scratch, copied by value
            size_t smem = 0;
            uint32_t tot = 0;
            for (int k = 0; k < m; k++) {
                const GridLaunch<R>& l = L[all[c0 + k]];
                P->ps[k] = l.gp;
                P->tile_base[k] = tot;
                tot += uint32_t(l.ntiles);
                smem = std::max(smem, l.smem);
            }
            P->tile_base[m] = tot;
            P->nsnap = m;
            P->counter = c->buf<uint32_t>("g" + std::to_string(gi++) + "ctr", 1);
            STPGPU_CUDA_TRY(cudaMemsetAsync(P->counter, 0, sizeof(uint32_t), main));
            if (class_ms)
                STPGPU_CUDA_TRY(cudaEventRecord(c->pev[0], main));
            const GridLaunch<R>& l0 = L[all[c0]];
            launch_group<R, COMP>(main, l0.kind,
                l0.tile_c | (B[all[c0]].persist ? kLayoutPersist : 0) | (l0.form == 2 ? kLayoutTaps : 0)
                    | (l0.form == 3 ? kLayoutRecs : 0),
                smem, *P, tot, capturing);
            nlaunch++;
            if (class_ms) {
                STPGPU_CUDA_TRY(cudaEventRecord(c->pev[1], main));
                STPGPU_CUDA_TRY(cudaEventSynchronize(c->pev[1]));
                float ms = 0.f;
                STPGPU_CUDA_TRY(cudaEventElapsedTime(&ms, c->pev[0], c->pev[1]));
                (*class_ms)[B[all[c0]].cls] += ms;
            }
        }
    }

    // ---- c2r + normalise per snapshot, scalars
    batch_fork(c, main);
    for (int i = 0; i < nb; i++) {
        c->stream = c->wstreams[i % K];
        c->ns = "b" + std::to_string(i) + "/";
        BatchSnap& b = B[i];
        finish_imager<R>(c, b.s, b.image_size, b.correction, G[i], dimg[i], nullptr, out_f32);
        BatchScalars* ds = c->buf<BatchScalars>("scal", 1);
        k_collect_scalars<<<1, 1, 0, c->stream>>>(G[i].d_total, G[i].d_ngood, G[i].d_nitems, G[i].d_err,
            G[i].d_plane_support ? G[i].d_plane_support : reinterpret_cast<const int*>(G[i].d_err),
            G[i].d_plane_support ? G[i].nplanes : 0, ds);
        STPGPU_CHECK_LAUNCH();
        STPGPU_CUDA_TRY(cudaMemcpyAsync(&scal[i], ds, sizeof(BatchScalars), cudaMemcpyDeviceToHost, c->stream));
        if (!device_ptrs)
            STPGPU_CUDA_TRY(cudaMemcpyAsync(b.image, dimg[i], (out_f32 ? 4 : 8) * size_t(b.image_size) * b.image_size,
                cudaMemcpyDeviceToHost, c->stream));
    }
    c->stream = main;
    c->ns = "";
    batch_join(c, main);
    return nlaunch;
}


template <typename R, int COMP>
void run_batch(stpgpu_context* c, const stpgpu_snapshot* sn, int nb, int precision, int out_f32, int device_ptrs,
    stpgpu_imager_info* infos, stpgpu_batch_info* bi)
{
    batch_streams(c);
    c->drop_single();
    std::vector<BatchSnap> B(nb);
    std::string sig;
    auto put = [&](const void* p, size_t n) { sig.append(reinterpret_cast<const char*>(p), n); };
    put(&precision, sizeof(int));
    put(&out_f32, sizeof(int));
    put(&device_ptrs, sizeof(int));
    for (int i = 0; i < nb; i++) {
        const stpgpu_snapshot& x = sn[i];
        BatchSnap& b = B[i];
        b.s = setup_from(&x.pars, &x.wproj, nullptr, b.image_size);
        if (x.pars.generate_beam)
            fail(STPGPU_ERR_UNSUPPORTED, "generate_beam is not supported by the batch path");
        if (b.image_size <= 0 || b.image_size > b.s.N || (b.image_size % 2) != 0)
            fail(STPGPU_ERR_INVALID_ARG, "snapshot " + std::to_string(i) + ": image_size must be even, > 0 and <= padded size");
        if (x.n_vis < 0 || (x.n_vis > 0 && (!x.vis || !x.weights || !x.uvw)) || !x.image)
            fail(STPGPU_ERR_INVALID_ARG, "snapshot " + std::to_string(i) + ": null buffer");
        if (x.vis_dtype != STPGPU_C128 && x.vis_dtype != STPGPU_C64)
            fail(STPGPU_ERR_INVALID_ARG, "snapshot " + std::to_string(i) + ": vis_dtype");
        b.correction = x.pars.gridding_correction;
        if (precision == STPGPU_FP32C)
            b.s.wide_fft = wide_fft_needed(b.s, b.image_size, b.correction) ? 1 : 0;
        b.vis = x.vis;
        b.c64 = x.vis_dtype == STPGPU_C64;
        b.wts = x.weights;
        b.uvw = x.uvw;
        b.n = x.n_vis;
        b.image = x.image;
        b.cls = size_class(b.s, precision) + "/batch";
        // W-planes without the |w| sort where they apply (as in single calls)
        b.s.wsel = b.s.nplanes > 0 && b.s.nplanes <= WSEL_MAXP && !b.s.wmedian && b.s.ntimesteps == 0
            && x.n_vis < (int64_t(1) << 31) && !c->wsel_off.count(b.cls);
        put(&b.s.wsel, sizeof(b.s.wsel));
        put(&x.pars, sizeof(x.pars));
        put(&x.wproj, sizeof(x.wproj));
        put(&x.n_vis, sizeof(x.n_vis));
        put(&x.vis_dtype, sizeof(x.vis_dtype));
        put(&x.vis, sizeof(void*));
        put(&x.weights, sizeof(void*));
        put(&x.uvw, sizeof(void*));
        put(&x.image, sizeof(void*));
    }
    if (sig != c->batch_sig) {
        for (auto w : c->wstreams)
            STPGPU_CUDA_TRY(cudaStreamSynchronize(w));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(c->stream));
        c->drop_graph();
        c->batch_sig = sig;
        c->batch_calls = 0;
    }
    c->batch_calls++;
    // pinned staging: scalars read back by the device + host scratch for the
    // by-value gridder parameter block
    const size_t need = pad256(sizeof(BatchScalars) * nb) + pad256(sizeof(BatchGridParams<R>)) + 4096;
    if (c->batch_host_cap < need) {
        if (c->batch_host) {
            for (auto w : c->wstreams)
                STPGPU_CUDA_TRY(cudaStreamSynchronize(w));
            STPGPU_CUDA_TRY(cudaStreamSynchronize(c->stream));
            c->drop_graph();
            cudaFreeHost(c->batch_host);
            c->batch_host = nullptr;
            c->batch_host_cap = 0;
        }
        STPGPU_CUDA_TRY(cudaMallocHost(&c->batch_host, need));
        c->batch_host_cap = need;
    }
    BatchScalars* scal = reinterpret_cast<BatchScalars*>(c->batch_host);
    unsigned char* hparams = reinterpret_cast<unsigned char*>(c->batch_host) + pad256(sizeof(BatchScalars) * nb);
    const bool saved_timing = c->timing;
    c->timing = false;
    struct Restore {
        stpgpu_context* c;
        cudaStream_t main;
        bool timing;
        ~Restore()
        {
            c->stream = main;
            c->ns = "";
            c->timing = timing;
        }
    } restore { c, c->stream, saved_timing };
    const cudaStream_t main = c->stream;
    int tuned = 0, glaunch = 0, graph = 0;
    g_launches = 0;
    if (device_ptrs && c->batch_exec) {
        // replay
        STPGPU_CUDA_TRY(cudaEventRecord(c->ev0, main));
        STPGPU_CUDA_TRY(cudaGraphLaunch(c->batch_exec, main));
        STPGPU_CUDA_TRY(cudaEventRecord(c->ev1, main));
        g_launches = c->batch_launches; // the replay runs the captured kernels
        graph = 1;
    } else {
        // tile autotuner: time both tile widths for classes not seen before
        std::vector<std::string> fresh;
        for (auto& b : B)
            if (int v; !c->tune_get(b.cls, v) && std::find(fresh.begin(), fresh.end(), b.cls) == fresh.end())
                fresh.push_back(b.cls);
        if (!fresh.empty()) {
            constexpr int NC = 12;
            const int layouts[NC] = { 32, 16, 32 | kLayoutPersist, 16 | kLayoutPersist, 32 | kLayoutTaps,
                16 | kLayoutTaps, 32 | kLayoutPersist | kLayoutTaps, 16 | kLayoutPersist | kLayoutTaps, 32 | kLayoutRecs,
                16 | kLayoutRecs, 32 | kLayoutPersist | kLayoutRecs, 16 | kLayoutPersist | kLayoutRecs };
            std::map<std::string, float> t[NC];
            for (int k = 0; k < 5; k++)
                if (!c->pev[k])
                    STPGPU_CUDA_TRY(cudaEventCreate(&c->pev[k]));
            for (int cand = 0; cand < NC; cand++) {
                for (auto& b : B) {
                    int lay = layouts[cand];
                    c->tune_get(b.cls, lay);
                    apply_layout(b, lay);
                }
                batch_enqueue<R, COMP>(c, B, out_f32, device_ptrs, false, scal, hparams, &t[cand]);
                STPGPU_CUDA_TRY(cudaStreamSynchronize(main));
            }
            static const bool log_tuning = std::getenv("STPGPU_LOG_TUNING") != nullptr;
            for (auto& cls : fresh) {
                int best = 0;
                for (int cand = 1; cand < NC; cand++)
                    if (t[cand][cls] < t[best][cls])
                        best = cand;
                c->tune_set(cls, layouts[best]);
                if (log_tuning)
                    std::fprintf(stderr,
                        "stpgpu gridder tuner: %s  32/16 cols %.3f/%.3f ms, persistent %.3f/%.3f ms, lane-per-tap"
                        " %.3f/%.3f ms, lane-per-tap persistent %.3f/%.3f ms, staged %.3f/%.3f ms, staged"
                        " persistent %.3f/%.3f ms -> %d%s%s\n",
                        cls.c_str(), double(t[0][cls]), double(t[1][cls]), double(t[2][cls]), double(t[3][cls]),
                        double(t[4][cls]), double(t[5][cls]), double(t[6][cls]), double(t[7][cls]),
                        double(t[8][cls]), double(t[9][cls]), double(t[10][cls]), double(t[11][cls]),
                        layouts[best] & 0xff, (layouts[best] & kLayoutPersist) ? " persistent" : "",
                        (layouts[best] & kLayoutRecs) ? " staged" : ((layouts[best] & kLayoutTaps) ? " lane-per-tap" : ""));
            }
            tuned = int(fresh.size());
        }
        for (auto& b : B) {
            int lay = TILE_C_DEFAULT;
            c->tune_get(b.cls, lay);
            apply_layout(b, lay);
        }
        bool capturable = true;
        for (auto& b : B)
            capturable = capturable && !large_support(b.s);
        if (device_ptrs && capturable && c->batch_calls >= 2 && tuned == 0) {
            // capture the batch (buffers, plans and tables exist from the previous call)
            STPGPU_CUDA_TRY(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
            try {
                glaunch = batch_enqueue<R, COMP>(c, B, out_f32, device_ptrs, true, scal, hparams, nullptr);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(main, &g);
                if (g)
                    cudaGraphDestroy(g);
                throw;
            }
            STPGPU_CUDA_TRY(cudaStreamEndCapture(main, &c->batch_graph));
            int zk = 0;
            c->batch_graph = memsets_to_kernels(c->batch_graph, &zk);
            g_launches += zk;
            c->batch_launches = g_launches;
            STPGPU_CUDA_TRY(cudaGraphInstantiate(&c->batch_exec, c->batch_graph, 0));
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev0, main));
            STPGPU_CUDA_TRY(cudaGraphLaunch(c->batch_exec, main));
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev1, main));
            graph = 1;
        } else {
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev0, main));
            glaunch = batch_enqueue<R, COMP>(c, B, out_f32, device_ptrs, false, scal, hparams, nullptr);
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev1, main));
        }
    }
    STPGPU_CUDA_TRY(cudaStreamSynchronize(main));
    for (int round = 0; round < 2; round++) {
        bool redo = false;
        for (int i = 0; i < nb; i++) {
            if (scal[i].err & 16u) { // the W-planes without the sort did not apply: the sorting path
                B[i].s.wsel = 0;
                c->wsel_off.insert(B[i].cls);
                redo = true;
            } else if (scal[i].err & 4u) { // long run of distinct |w| in the 24-bit sort: the 64-bit sort
                B[i].s.full_wsort = 1;
                redo = true;
            }
        }
        if (!redo)
            break;
        c->drop_graph();
        c->batch_calls = 0;
        c->batch_sig.clear();
        STPGPU_CUDA_TRY(cudaEventRecord(c->ev0, main));
        glaunch = batch_enqueue<R, COMP>(c, B, out_f32, device_ptrs, false, scal, hparams, nullptr);
        STPGPU_CUDA_TRY(cudaEventRecord(c->ev1, main));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(main));
        graph = 0;
    }
    float ms = 0.f;
    STPGPU_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    for (int i = 0; i < nb; i++) {
        if (scal[i].err & ~4u)
            fail(STPGPU_ERR_DEVICE, "snapshot " + std::to_string(i) + ": gridder reported internal error flags "
                    + std::to_string(scal[i].err));
        if (infos) {
            stpgpu_imager_info& f = infos[i];
            std::memset(&f, 0, sizeof(f));
            f.sample_grid_total = scal[i].total;
            f.n_good_vis = int64_t(scal[i].ngood);
            f.n_grid_items = scal[i].nitems;
            f.padded_image_size = B[i].s.N;
            f.num_wplanes = B[i].s.nplanes;
            f.max_plane_support = scal[i].max_support;
            f.image_size = scal[i].total > 0.0 ? B[i].image_size : 0;
            f.flags = B[i].s.wide_fft ? 1 : 0;
        }
    }
    if (bi) {
        std::memset(bi, 0, sizeof(*bi));
        bi->device_ms = ms;
        bi->graph = graph;
        bi->gridder_launches = glaunch;
        bi->tuned_classes = tuned;
        bi->n_launches = g_launches;
    }
}

// ------------------------------------------------------------------ source finder

// Exact k-th order statistic (0-based) by 16-bit radix select.
template <typename T>
double select_kth(stpgpu_context* c, const T* x, int64_t n, unsigned long long k)
{
    cudaStream_t st = c->stream;
    unsigned int* hist = c->buf<unsigned int>("rsel_hist", 65536);
    unsigned long long* state = c->buf<unsigned long long>("rsel_state", 3);
    unsigned long long h0[3] = { k, 0ull, 0ull };
    STPGPU_CUDA_TRY(cudaMemcpyAsync(state, h0, sizeof(h0), cudaMemcpyHostToDevice, st));
    unsigned long long* hs = c->host_stage<unsigned long long>(3);
    for (int pass = 3; pass >= 0; pass--) {
        const int shift = pass * 16;
        STPGPU_CUDA_TRY(cudaMemsetAsync(hist, 0, sizeof(unsigned int) * 65536, st));
        // prefix/mask are read on the host after each pass
        STPGPU_CUDA_TRY(cudaMemcpyAsync(hs, state, sizeof(h0), cudaMemcpyDeviceToHost, st));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
        k_radix_hist<T><<<std::min<unsigned>(grid1d(n, SF_THREADS), 148 * 16), SF_THREADS, 0, st>>>(x, n, hs[1],
            hs[2], shift, hist);
        STPGPU_CHECK_LAUNCH();
        k_radix_pick<<<1, 1024, 0, st>>>(hist, shift, state);
        STPGPU_CHECK_LAUNCH();
    }
    STPGPU_CUDA_TRY(cudaMemcpyAsync(hs, state, sizeof(h0), cudaMemcpyDeviceToHost, st));
    STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
    // key -> double
    const unsigned long long key = hs[1];
    const unsigned long long u = (key >> 63) ? (key & 0x7fffffffffffffffull) : ~key;
    double v;
    std::memcpy(&v, &u, sizeof(v));
    return v;
}

// mat_median_exact (matrix_math.cpp:20-48)
template <typename T>
double median_exact(stpgpu_context* c, const T* x, int64_t n)
{
    const unsigned long long k = (unsigned long long)(n / 2);
    const double v1 = select_kth(c, x, n, k);
    if (n & 1)
        return v1;
    const double v2 = select_kth(c, x, n, k - 1);
    return (v1 + v2) / 2;
}

// Gaussian2dParams::convert_to_constrained_parameters (fitting.cpp:32-57)
void constrain(double* g)
{
    const double half_pi = M_PI / 2.0;
    g[3] = std::fabs(g[3]);
    g[4] = std::fabs(g[4]);
    if (g[3] < g[4]) {
        std::swap(g[3], g[4]);
        g[5] += half_pi;
    }
    double t = std::fmod(g[5], M_PI);
    if (t <= -half_pi)
        t += M_PI;
    else if (t > half_pi)
        t -= M_PI;
    g[5] = t;
}

// IslandParams::estimate_moments_fit (sourcefind.cpp:691-717)
void moments_fit(int sign, double extremum, const double* mb, double rms, double ana_sigma, double* g)
{
    const double xx = mb[2], yy = mb[3], xy = mb[4];
    const double w1 = (xx + yy) / 2.0;
    const double w2 = std::sqrt(((xx - yy) * (xx - yy) / 4) + xy * xy);
    const double tmaj = w1 + w2, tmin = w1 - w2;
    const double thr = ana_sigma * rms;
    const double ratio = sign * extremum / thr;
    const double scale = 1.0 - std::log(ratio) / (ratio - 1.0);
    double theta = 0.5 * std::atan(2.0 * xy / (xx - yy));
    if (theta * xy < 0.0)
        theta += M_PI / 2.0;
    g[0] = extremum;
    g[1] = mb[0];
    g[2] = mb[1];
    g[3] = std::sqrt(tmaj / scale);
    g[4] = std::sqrt(tmin / scale);
    g[5] = theta;
    constrain(g);
}

// k_seg_sort_big uses SEG_BIG indices of dynamic shared memory (more than the
// default 48 KB): raise its limit once per device.
void set_seg_sort_smem()
{
    static std::atomic<uint64_t> done { 0 };
    int dev = 0;
    STPGPU_CUDA_TRY(cudaGetDevice(&dev));
    const uint64_t bit = uint64_t(1) << (dev & 63);
    if (done.load() & bit)
        return;
    STPGPU_CUDA_TRY(cudaFuncSetAttribute(k_seg_sort_big, cudaFuncAttributeMaxDynamicSharedMemorySize,
        int(SEG_BIG * sizeof(uint32_t))));
    done.fetch_or(bit);
}

// Device state of one source-finder call: labeller counters, pass tickets,
// statistics and the clipping state, cleared by one memset per call.
struct SfState {
    uint32_t misc[8]; // CclBufs::misc, then the valid-label count [4] and the island count [5]
    unsigned int tickets[4];
    uint32_t seg[3]; // label analysis: segment allocation cursor, labels with entries, labels for the one-block sort
    SfStats st;
    ClipState cs;
};

// Blocks of the fused statistics kernel for T on the context's device (the
// cooperative grid: one block per SM); 0 when it cannot be launched
// cooperatively.
template <typename T>
int sf_stats_grid(stpgpu_context* c)
{
    static std::mutex mu;
    static std::map<int, int> grid;
    std::lock_guard<std::mutex> lk(mu);
    auto it = grid.find(c->device);
    if (it != grid.end())
        return it->second;
    int coop = 0, sms = 0, per_sm = 0;
    STPGPU_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
    STPGPU_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
    STPGPU_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sf_stats<T>, SF_STATS_THREADS, 0));
    const int g = coop ? std::min(per_sm, 1) * sms : 0;
    grid[c->device] = g;
    return g;
}

// Images of at least this many samples take the fused statistics kernel;
// smaller ones the pass kernels.
constexpr int64_t kSfFusedMin = int64_t(1) << 16;

// The pass kernels for every image when STPGPU_SF_STATS=passes.
bool sf_passes_forced()
{
    const char* e = std::getenv("STPGPU_SF_STATS");
    return e && std::strcmp(e, "passes") == 0;
}

// The statistics' working buffers at the sizes enqueue_stats asks for, so
// that a call sizes them before it looks at its graph signature.
template <typename T>
void size_stats_buffers(stpgpu_context* c, int64_t n, const stpgpu_sf_pars& p)
{
    const bool est = !(std::fabs(p.rms_est) > 0.0);
    const int grid = sf_stats_grid<T>(c);
    if (grid > 0) {
        const int64_t G = int64_t(grid) * SF_STATS_THREADS;
        c->buf<double>("sf_part_fused", 8 * size_t(grid));
        if (est)
            c->buf<T>("sf_clip_lists", size_t(sf_band_cap(n, G)) * size_t(G));
    }
    const unsigned nb = std::min<unsigned>(grid1d(n, SF_THREADS), 148 * SF_STREAM_BLOCKS);
    c->buf<double>("sf_part", 3 * size_t(nb));
    c->buf<unsigned long long>("sf_bins", BINS_N + 2);
}

// Statistics and thresholds (sourcefind.cpp:280-301) enqueued into s->st;
// only the exact median (NTHELEMENT, BINMEDIAN, or exact = the binned
// median's fallback) waits on the host.  With `fused` (16-byte aligned
// images of at least kSfFusedMin samples) one cooperative launch of
// k_sf_stats does the passes; otherwise one kernel per pass.
template <typename T>
void enqueue_stats(stpgpu_context* c, const T* x, int64_t n, const stpgpu_sf_pars& p, SfState* s, bool exact,
    bool fused)
{
    cudaStream_t st = c->stream;
    const bool est = !(std::fabs(p.rms_est) > 0.0);
    const int grid = fused ? sf_stats_grid<T>(c) : 0;
    if (grid > 0 && n >= kSfFusedMin && (reinterpret_cast<uintptr_t>(x) & 15) == 0 && !sf_passes_forced()) {
        int do_sum = est, do_hist = 0;
        switch (p.median_method) {
        case STPGPU_ZEROMEDIAN:
            break;
        case STPGPU_BINAPPROX:
            if (!exact) {
                do_sum = 1;
                do_hist = 1;
                break;
            }
            [[fallthrough]];
        case STPGPU_BINMEDIAN:
            do_sum = 1;
            [[fallthrough]];
        case STPGPU_NTHELEMENT:
            k_sf_set_median<<<1, 1, 0, st>>>(&s->st, median_exact(c, x, n));
            STPGPU_CHECK_LAUNCH();
            break;
        default:
            fail(STPGPU_ERR_INVALID_ARG, "unknown median method");
        }
        const int64_t G = int64_t(grid) * SF_STATS_THREADS;
        int cap = est ? sf_band_cap(n, G) : 0;
        double* part = c->buf<double>("sf_part_fused", 8 * size_t(grid));
        unsigned long long* bins = c->buf<unsigned long long>("sf_bins", BINS_N + 2);
        T* cand = est ? c->buf<T>("sf_clip_lists", size_t(cap) * size_t(G)) : nullptr;
        int iters = est ? p.sigma_clip_iters : 0;
        double rms = p.rms_est, ana = p.analysis_n_sigma, det = p.detection_n_sigma;
        const T* xa = x;
        SfStats* sta = &s->st;
        ClipState* csa = &s->cs;
        unsigned int* bar = &s->tickets[3];
        void* args[] = { (void*)&xa, (void*)&n, (void*)&sta, (void*)&csa, (void*)&part, (void*)&bins, (void*)&cand,
            (void*)&cap, (void*)&bar, (void*)&do_sum, (void*)&do_hist, (void*)&iters, (void*)&rms, (void*)&ana,
            (void*)&det };
        STPGPU_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_sf_stats<T>, dim3(grid), dim3(SF_STATS_THREADS), args,
            0, st));
        return;
    }
    const unsigned nb = std::min<unsigned>(grid1d(n, SF_THREADS), 148 * SF_STREAM_BLOCKS);
    double* part = c->buf<double>("sf_part", 3 * size_t(nb));
    unsigned long long* bins = c->buf<unsigned long long>("sf_bins", BINS_N + 2);
    auto sum_sq = [&](bool with_bins) {
        k_sum_sq<T><<<nb, SF_THREADS, 0, st>>>(x, n, part, &s->tickets[0], &s->st, with_bins ? bins : nullptr);
        STPGPU_CHECK_LAUNCH();
    };
    auto set_median = [&](double m) {
        k_sf_set_median<<<1, 1, 0, st>>>(&s->st, m);
        STPGPU_CHECK_LAUNCH();
    };
    switch (p.median_method) {
    case STPGPU_ZEROMEDIAN: // the state starts at zero
        if (est)
            sum_sq(false);
        break;
    case STPGPU_BINAPPROX:
        if (!exact) {
            sum_sq(true);
            k_hist<T><<<nb, SF_THREADS, 0, st>>>(x, n, &s->st, bins, &s->tickets[1]);
            STPGPU_CHECK_LAUNCH();
            break;
        }
        [[fallthrough]];
    case STPGPU_BINMEDIAN: // successive binning ends in nth_element: the exact median
        sum_sq(false);
        set_median(median_exact(c, x, n));
        break;
    case STPGPU_NTHELEMENT:
        set_median(median_exact(c, x, n));
        if (est)
            sum_sq(false);
        break;
    default:
        fail(STPGPU_ERR_INVALID_ARG, "unknown median method");
    }
    if (est) {
        k_clip_init<<<1, 1, 0, st>>>(&s->cs, &s->st, double(n), 3.0);
        STPGPU_CHECK_LAUNCH();
        for (int it = 0; it < p.sigma_clip_iters; it++) {
            k_clip_pass<T><<<nb, SF_THREADS, 0, st>>>(x, n, &s->st, &s->cs, part, &s->tickets[2], 3.0);
            STPGPU_CHECK_LAUNCH();
        }
    }
    k_sf_thresholds<<<1, 1, 0, st>>>(&s->st, est ? &s->cs : nullptr, p.rms_est, p.analysis_n_sigma,
        p.detection_n_sigma);
    STPGPU_CHECK_LAUNCH();
}

// Labeller buffers for n pixels in ccl_chunks(n) chunks.
struct CclBufs {
    uint8_t* cls; // ccl_chunks(n) * CCL_CHUNK bytes (background padding past n)
    uint32_t* P; // n union-find parents (foreground keys only)
    uint32_t* R; // n: label number of each root
    uint32_t* cnt; // 3 rows of ccl_chunks(n) + 1: positive roots, negative roots, foreground keys per chunk
    uint32_t* off; // their exclusive scans, same layout
    uint32_t* misc; // [0..2] the three totals, [3] union-find step-bound flag (zero before the call)
    uint32_t* fgl; // n: foreground keys in scan order, or null
    int32_t* L; // n: label map in memory order, or null
};

inline int64_t ccl_chunks(int64_t n) { return (n + CCL_CHUNK - 1) / CCL_CHUNK; }

// Enqueues the labeller (ccl.h:19-773 semantics, see the kernels) on st.
// Counts its launches; makes no allocation and throws nothing.
template <typename T>
cudaError_t ccl_enqueue(cudaStream_t st, const T* img, const CclGeom& g, const double* thr, double tp, double tn,
    int findneg, int conn4, int slice, const CclBufs& b)
{
    const int64_t n = int64_t(g.rows) * g.cols;
    const int64_t nch = ccl_chunks(n), npad = nch * CCL_CHUNK;
    const int stride = int(nch + 1);
    unsigned* err = b.misc + 3;
    if (g.rows % 4 == 0 && (reinterpret_cast<uintptr_t>(img) & 15) == 0) {
        const int64_t nu = npad / CCL_KPT;
        k_ccl_init16<T><<<unsigned(std::min<int64_t>(ceil_div(nu, SF_THREADS), 148 * 4)), SF_THREADS, 0, st>>>(img,
            g, thr, tp, tn, findneg, n / 4, nu, reinterpret_cast<uint4*>(b.cls), reinterpret_cast<uint4*>(b.P));
    } else {
        if (npad > n) {
            const cudaError_t e = cudaMemsetAsync(b.cls + n, 0, size_t(npad - n), st);
            if (e != cudaSuccess)
                return e;
        }
        k_ccl_init<T><<<grid1d(n, 256), 256, 0, st>>>(img, g, thr, tp, tn, findneg, b.cls, b.P);
    }
    k_ccl_union<<<unsigned(nch), SF_THREADS, 0, st>>>(b.cls, g, conn4, slice, b.P, err);
    k_ccl_flatten<<<unsigned(nch), SF_THREADS, 0, st>>>(b.cls, b.P, b.cnt, stride, err);
    k_scan_rows<<<3, 1024, 0, st>>>(b.cnt, b.off, int(nch), stride, b.misc);
    k_ccl_rank<<<unsigned(nch), SF_THREADS, 0, st>>>(b.cls, b.P, b.off, stride, b.R, b.fgl);
    g_launches += 5;
    if (b.L) {
        if (g.rows % 4 == 0 && (reinterpret_cast<uintptr_t>(b.L) & 15) == 0) {
            const int64_t ng = n / 4;
            k_ccl_label16<<<unsigned(std::min<int64_t>(ceil_div(ceil_div(ng, 4), SF_THREADS), 148 * 8)), SF_THREADS,
                0, st>>>(b.cls, b.P, b.R, g, ng, b.L);
        } else {
            k_ccl_label<<<grid1d(n, 256), 256, 0, st>>>(b.cls, b.P, b.R, g, b.L);
        }
        g_launches++;
    }
    return cudaGetLastError();
}

// write_labels: fill the label map (d_labels, or the context's "ccl_L"
// buffer when d_labels is null).
template <typename T>
void run_source_find(stpgpu_context* c, const T* d_img, int rows, int cols, const stpgpu_sf_pars& p, int32_t* d_labels,
    bool write_labels, std::vector<stpgpu_island>& islands, stpgpu_sf_info& info)
{
    if (rows <= 0 || cols <= 0 || (rows % 2) || (cols % 2))
        fail(STPGPU_ERR_INVALID_ARG, "image dimensions must be positive and even (ccl.h:116-117)");
    if (rows > 65536 || cols > 65536 || int64_t(rows) * cols >= (int64_t(1) << 32))
        fail(STPGPU_ERR_INVALID_ARG, "image too large for the labeler (ccl.h:118-119)");
    cudaStream_t st = c->stream;
    const int64_t n = int64_t(rows) * cols;
    // ---- connected components
    const CclGeom geom { rows, cols, rows / 2, cols / 2 };
    const int64_t nch = ccl_chunks(n);
    CclBufs cb;
    cb.cls = c->buf<uint8_t>("ccl_cls", size_t(nch) * CCL_CHUNK);
    cb.P = c->buf<uint32_t>("ccl_P", n);
    cb.R = c->buf<uint32_t>("ccl_R", n);
    cb.cnt = c->buf<uint32_t>("ccl_cnt", 3 * size_t(nch + 1));
    cb.off = c->buf<uint32_t>("ccl_off", 3 * size_t(nch + 1));
    cb.fgl = c->buf<uint32_t>("ccl_fgl", n);
    cb.L = write_labels ? (d_labels ? d_labels : c->buf<int32_t>("ccl_L", n)) : nullptr;
    SfState* sfs = c->buf<SfState>("sf_state", 1);
    cb.misc = sfs->misc;
    const int slice = p.ccl_slice_cols > 0 ? p.ccl_slice_cols : std::max(2, cols / 8);

    // ---- extrema, detection filter, moments (sourcefind.cpp:342-628) over
    // the foreground list, enqueued behind the labeller before its counts are
    // known: the buffers are sized by capacities (remembered per context),
    // and a call whose counts exceed them runs this stage again
    constexpr bool packed = sizeof(T) == 4;
    constexpr int kFirst = 512; // island records read back with the counts
    const unsigned G = 148 * 4; // grid of the label-analysis loops
    const uint32_t split_m = uint32_t(cols / 2) * uint32_t(rows);
    int32_t* zero_map = p.generate_labelmap ? cb.L : nullptr;
    uint32_t* nvalid = cb.misc + 4;
    uint32_t* nisl = cb.misc + 5;
    uint32_t* nvk = cb.misc + 6; // valid entries
    uint32_t* sort_overflow = cb.misc + 7;
    uint32_t lcap = uint32_t(std::min<int64_t>(n, std::max<int64_t>(c->sf_label_cap, std::max<int64_t>(65536, n / 64))));
    uint32_t fcap = uint32_t(std::min<int64_t>(n, std::max<int64_t>(c->sf_fg_cap, std::max<int64_t>(131072, n / 16))));
    unsigned long long *ext = nullptr, *eidx = nullptr, *vkeys = nullptr;
    double* mom = nullptr;
    int* ns = nullptr;
    uint32_t *sb = nullptr, *se = nullptr, *sp = nullptr, *fcode = nullptr, *fm = nullptr, *v1 = nullptr;
    uint32_t *cursor = nullptr, *slots = nullptr, *bigl = nullptr, *listed = nullptr;
    IslandRaw* raw = nullptr;
    auto size_buffers = [&] {
        // per label: extremum keys (single precision: value-and-index keys),
        // first indices, moments, sample counts, list segments; per list
        // entry: label code, memory index, valid keys, sorted memory indices
        ext = c->buf<unsigned long long>("sf_ext", lcap);
        eidx = c->buf<unsigned long long>("sf_eidx", lcap);
        mom = c->buf<double>("sf_mom", 6 * size_t(lcap));
        ns = c->buf<int>("sf_ns", lcap);
        sb = c->buf<uint32_t>("fg_sb", lcap);
        se = c->buf<uint32_t>("fg_se", lcap);
        sp = c->buf<uint32_t>("fg_sp", lcap);
        raw = c->buf<IslandRaw>("sf_raw", std::max<uint32_t>(lcap, kFirst));
        fcode = c->buf<uint32_t>("fg_code", fcap);
        fm = c->buf<uint32_t>("fg_m", fcap);
        vkeys = c->buf<unsigned long long>("fg_vkeys", fcap);
        v1 = c->buf<uint32_t>("fg_v1", fcap);
        cursor = c->buf<uint32_t>("fg_cur", lcap);
        slots = c->buf<uint32_t>("fg_slots", fcap);
        bigl = c->buf<uint32_t>("fg_big", lcap);
        listed = c->buf<uint32_t>("fg_listed", lcap);
    };
    auto moments_and_islands = [&](const FgSizes& z) {
        k_label_sums<T><<<G, 128, 0, st>>>(z, d_img, rows, cols, v1, sb, se, sp, mom, ns);
        STPGPU_CHECK_LAUNCH();
        k_islands<packed><<<G, 256, 0, st>>>(z, &sfs->st, ext, eidx, ns, mom, p.source_min_area, nvalid, nisl, raw);
        STPGPU_CHECK_LAUNCH();
    };
    auto enqueue_analysis = [&] {
        const FgSizes z { cb.misc, lcap, fcap };
        k_fg_init<packed><<<G, 256, 0, st>>>(z, &sfs->st, ext, packed ? nullptr : eidx, sb, se, sp);
        STPGPU_CHECK_LAUNCH();
        k_fg_gather<T, packed><<<G, 256, 0, st>>>(z, d_img, cb.cls, cb.P, cb.R, geom, cb.fgl, fcode, fm, ext);
        STPGPU_CHECK_LAUNCH();
        if constexpr (!packed) {
            k_fg_extrema_idx<T><<<G, 256, 0, st>>>(z, &sfs->st, d_img, fcode, fm, ext, eidx);
            STPGPU_CHECK_LAUNCH();
        }
        k_fg_keys<packed><<<G, 256, 0, st>>>(z, &sfs->st, fcode, fm, ext, vkeys, nvk, zero_map, se);
        STPGPU_CHECK_LAUNCH();
        // ordered (deterministic) moments: each valid label's entries in a
        // range of their own, ordered by list position (one warp per label,
        // one block for the large ones), per-label sums in memory order;
        // island records appended in any order
        k_seg_alloc<<<G, 256, 0, st>>>(z, sb, se, cursor, &sfs->seg[0], listed);
        STPGPU_CHECK_LAUNCH();
        k_seg_scatter<<<G, 256, 0, st>>>(vkeys, nvk, cursor, slots);
        STPGPU_CHECK_LAUNCH();
        k_seg_sort<<<G, 256, 0, st>>>(listed, &sfs->seg[1], sb, se, slots, fm, split_m, v1, sp, bigl, &sfs->seg[2]);
        STPGPU_CHECK_LAUNCH();
        set_seg_sort_smem();
        k_seg_sort_big<<<64, 1024, SEG_BIG * sizeof(uint32_t), st>>>(sb, se, slots, fm, split_m, v1, sp, bigl,
            &sfs->seg[2], sort_overflow);
        STPGPU_CHECK_LAUNCH();
        moments_and_islands(z);
    };
    // everything, then one read-back: state (statistics, counts, flags) and
    // the first island records
    unsigned char* hb = c->host_stage<unsigned char>(sizeof(SfState) + 64 + sizeof(IslandRaw) * size_t(kFirst));
    SfState* hstate = reinterpret_cast<SfState*>(hb);
    IslandRaw* hfirst = reinterpret_cast<IslandRaw*>(hb + ((sizeof(SfState) + 63) / 64) * 64);
    // the state and the first island records (as many as the call found, up
    // to kFirst) written by one kernel straight into the page-locked stage
    static_assert(sizeof(SfState) % 4 == 0 && (sizeof(IslandRaw) * kFirst) % 16 == 0, "copy-out units");
    auto enqueue_copy_out = [&] {
        k_copy_out<<<unsigned((sizeof(IslandRaw) * kFirst / 16 + 255) / 256), 256, 0, st>>>(
            reinterpret_cast<const uint32_t*>(sfs), c->host_stage_dev(reinterpret_cast<uint32_t*>(hstate)),
            int(sizeof(SfState) / 4), reinterpret_cast<const uint4*>(raw),
            c->host_stage_dev(reinterpret_cast<uint4*>(hfirst)), int(sizeof(IslandRaw) * kFirst / 16),
            int(offsetof(SfState, misc) / 4) + 5, int(sizeof(IslandRaw)));
        STPGPU_CHECK_LAUNCH();
    };
    auto read_back_state = [&] {
        enqueue_copy_out();
        STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
    };
    size_buffers();
    auto enqueue_attempt = [&](bool exact_median, bool fused_stats) {
        static_assert(sizeof(SfState) % 4 == 0, "SfState in 32-bit words");
        zero_words(st, { { sfs, int64_t(sizeof(SfState) / 4) } });
        enqueue_stats<T>(c, d_img, n, p, sfs, exact_median, fused_stats);
        STPGPU_CUDA_TRY(ccl_enqueue<T>(st, d_img, geom, sfs->st.thr, 0.0, 0.0, p.find_negative_sources,
            p.ccl_4connectivity, slice, cb));
        enqueue_analysis();
        enqueue_copy_out();
    };
    // The first attempt of a call identical to the previous one (same
    // buffers, sizes, parameters and capacities, no reallocation since)
    // replays a CUDA graph of it; the second such call captures it.  Calls
    // whose median needs the host (NTHELEMENT, BINMEDIAN) run eagerly, as does
    // every call after a capture that the runtime refused.
    size_stats_buffers<T>(c, n, p);
    std::string sig;
    if (!c->timing && !c->sf_graph_off
        && (p.median_method == STPGPU_ZEROMEDIAN || p.median_method == STPGPU_BINAPPROX)) {
        auto put = [&](const void* q, size_t nb) { sig.append(reinterpret_cast<const char*>(q), nb); };
        const int tsize = int(sizeof(T));
        const int forced = sf_passes_forced() ? 1 : 0;
        const int wl = write_labels ? 1 : 0;
        put(&tsize, sizeof(tsize));
        put(&rows, sizeof(rows));
        put(&cols, sizeof(cols));
        put(&p, sizeof(p));
        put(&wl, sizeof(wl));
        put(&forced, sizeof(forced));
        put(&lcap, sizeof(lcap));
        put(&fcap, sizeof(fcap));
        put(&c->buf_gen, sizeof(c->buf_gen));
        const void* ptrs[4] = { d_img, d_labels, hb, reinterpret_cast<const void*>(st) };
        put(ptrs, sizeof(ptrs));
    }
    const bool repeat = !sig.empty() && sig == c->sf_sig;
    if (!repeat) {
        c->drop_sf_graph();
        c->sf_sig = sig;
    }
    bool exact = false, fused = true;
    for (int attempt = 0; attempt < 3; attempt++) {
        // again when the binned median does not apply (the exact median), or
        // when the fused statistics kernel gave up at a barrier (the pass
        // kernels)
        if (attempt == 0 && repeat && c->sf_exec) {
            STPGPU_CUDA_TRY(cudaGraphLaunch(c->sf_exec, st));
            g_launches += c->sf_launches;
        } else if (attempt == 0 && repeat) {
            const int before = g_launches;
            bool captured = false;
            STPGPU_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_attempt(false, true);
                STPGPU_CUDA_TRY(cudaStreamEndCapture(st, &c->sf_graph));
                STPGPU_CUDA_TRY(cudaGraphInstantiate(&c->sf_exec, c->sf_graph, 0));
                captured = true;
            } catch (const Error&) {
                cudaGraph_t dead = nullptr;
                cudaStreamEndCapture(st, &dead); // ends a capture still open; fails harmlessly otherwise
                if (dead)
                    cudaGraphDestroy(dead);
                (void)cudaGetLastError();
                c->drop_sf_graph();
                c->sf_graph_off = true;
            }
            if (captured) {
                c->sf_launches = g_launches - before;
                STPGPU_CUDA_TRY(cudaGraphLaunch(c->sf_exec, st));
            } else {
                g_launches = before;
                enqueue_attempt(false, true);
            }
        } else {
            enqueue_attempt(exact, fused);
        }
        STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
        if (hstate->st.stats_err && fused) {
            fused = false;
            continue;
        }
        if (hstate->st.need_exact && !exact) {
            exact = true;
            continue;
        }
        break;
    }
    if (hstate->st.stats_err)
        fail(STPGPU_ERR_DEVICE, "source-finder statistics failed");
    if (hstate->misc[3])
        fail(STPGPU_ERR_DEVICE, "labeler gave up (union-find step bound)");
    const int np = int(hstate->misc[0]), nneg = int(hstate->misc[1]), nfg = int(hstate->misc[2]);
    const int nl = std::max(1, np + nneg);
    if (uint32_t(np + nneg) > lcap || uint32_t(nfg) > fcap) {
        // counts beyond the capacities: larger buffers, the stage again
        lcap = uint32_t(std::max<int64_t>(lcap, np + nneg + (np + nneg) / 4));
        fcap = uint32_t(std::max<int64_t>(fcap, nfg + nfg / 4));
        lcap = uint32_t(std::min<int64_t>(lcap, n));
        fcap = uint32_t(std::min<int64_t>(fcap, n));
        size_buffers();
        STPGPU_CUDA_TRY(cudaMemsetAsync(cb.misc + 4, 0, 4 * sizeof(uint32_t), st));
        STPGPU_CUDA_TRY(cudaMemsetAsync(sfs->seg, 0, sizeof(sfs->seg), st));
        enqueue_analysis();
        read_back_state();
    }
    c->sf_label_cap = std::max<uint32_t>(c->sf_label_cap, lcap);
    c->sf_fg_cap = std::max<uint32_t>(c->sf_fg_cap, fcap);
    if (hstate->misc[7]) {
        // a label with more valid entries than the one-block sort holds:
        // sort all entries with the multi-block sort, then sums and islands
        // again
        const uint32_t nv = hstate->misc[6];
        int end_bit = 33;
        while (end_bit < 64 && (uint64_t(1) << (end_bit - 32)) <= uint64_t(nl))
            end_bit++;
        unsigned long long* vk2 = c->buf<unsigned long long>("fg_vkeys2", nv);
        size_t tb = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, tb, vkeys, vk2, int(nv), 0, end_bit, st);
        void* tmp = c->buf<unsigned char>("cubtmp_sf", tb);
        if (cub::DeviceRadixSort::SortKeys(tmp, tb, vkeys, vk2, int(nv), 0, end_bit, st) != cudaSuccess)
            fail(STPGPU_ERR_CUDA, "label sort failed");
        k_seg_mark<<<grid1d(nv, 256), 256, 0, st>>>(vk2, nv, fm, split_m, v1, sb, se, sp);
        STPGPU_CHECK_LAUNCH();
        STPGPU_CUDA_TRY(cudaMemsetAsync(cb.misc + 4, 0, 2 * sizeof(uint32_t), st));
        moments_and_islands(FgSizes { cb.misc, lcap, fcap });
        read_back_state();
    }
    const SfState h = *hstate;
    info.bg_level = h.st.median;
    info.rms_est = h.st.rms;
    info.mean = h.st.mean;
    info.sigma = h.st.sigma;
    const double rms = h.st.rms;
    info.n_labels_pos = np;
    info.n_labels_neg = nneg;
    const int first = std::min(nl, kFirst);
    const uint32_t* fit_pix = h.misc[6] > 0 ? v1 : nullptr;
    const int nis = int(h.misc[5]);
    info.n_valid_labels = int(h.misc[4]);
    info.n_islands = nis;
    std::vector<IslandRaw> hr(nis);
    std::copy(hfirst, hfirst + std::min(nis, first), hr.begin());
    if (nis > first) {
        STPGPU_CUDA_TRY(cudaMemcpyAsync(hr.data() + first, raw + first, sizeof(IslandRaw) * (nis - first),
            cudaMemcpyDeviceToHost, st));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
    }
    // label order: positives by label, then negatives
    std::sort(hr.begin(), hr.end(), [](const IslandRaw& a, const IslandRaw& b) {
        const bool na = a.label < 0, nb = b.label < 0;
        if (na != nb)
            return nb;
        return std::abs(a.label) < std::abs(b.label);
    });
    islands.resize(nis);
    const int vs = rows / 2, hs = cols / 2;
    for (int i = 0; i < nis; i++) {
        const IslandRaw& r = hr[i];
        stpgpu_island& o = islands[i];
        std::memset(&o, 0, sizeof(o));
        o.label_idx = r.label;
        o.sign = r.label < 0 ? -1 : 1;
        o.extremum_val = r.extremum_val;
        const int row = int(r.extremum_idx % rows), col = int(r.extremum_idx / rows);
        o.extremum_y_idx = row < vs ? row + vs : row - vs; // sourcefind.cpp:243-244
        o.extremum_x_idx = col < hs ? col + hs : col - hs;
        o.num_samples = r.num_samples;
        // moment normalisation (sourcefind.cpp:591-604)
        const double* a = r.mom;
        double mb[5];
        mb[0] = a[0] / a[5];
        mb[1] = a[1] / a[5];
        mb[2] = a[2] / a[5] - mb[0] * mb[0];
        mb[3] = a[3] / a[5] - mb[1] * mb[1];
        mb[4] = a[4] / a[5] - mb[0] * mb[1];
        moments_fit(o.sign, o.extremum_val, mb, rms, p.analysis_n_sigma, o.moments_fit);
    }
    if (p.gaussian_fitting && nis > 0) {
        // least-squares 2-D Gaussian per island (sourcefind.cpp:719-866): islands of one or two pixels keep
        // (extremum, 0, ...); the others start from the moments fit, unset widths as 1
        std::vector<int> keys, which;
        std::vector<double> init;
        for (int i = 0; i < nis; i++) {
            stpgpu_island& o = islands[i];
            if (o.num_samples < 3) {
                o.leastsq_fit[0] = o.extremum_val;
                continue;
            }
            const int l = o.label_idx;
            keys.push_back(l > 0 ? l - 1 : np + (-l - 1));
            which.push_back(i);
            const double* m = o.moments_fit;
            const double g[6] = { m[0], m[1], m[2], m[3] > 0.0 ? m[3] : 1.0, m[4] > 0.0 ? m[4] : 1.0, m[5] };
            init.insert(init.end(), g, g + 6);
        }
        const int nfit = int(keys.size());
        if (nfit > 0 && fit_pix) {
            int* dkeys = c->buf<int>("fit_keys", nfit);
            double* dinit = c->buf<double>("fit_init", 6 * size_t(nfit));
            double* dout = c->buf<double>("fit_out", 6 * size_t(nfit));
            int* dit = c->buf<int>("fit_iter", nfit);
            STPGPU_CUDA_TRY(cudaMemcpyAsync(dkeys, keys.data(), sizeof(int) * nfit, cudaMemcpyHostToDevice, st));
            STPGPU_CUDA_TRY(cudaMemcpyAsync(dinit, init.data(), sizeof(double) * 6 * nfit, cudaMemcpyHostToDevice, st));
            k_gauss_fit<T><<<nfit, 32, 0, st>>>(d_img, rows, cols, fit_pix, sb, se, sp, dkeys, dinit, nfit, dout, dit);
            STPGPU_CHECK_LAUNCH();
            std::vector<double> out(6 * size_t(nfit));
            std::vector<int> its(nfit);
            STPGPU_CUDA_TRY(cudaMemcpyAsync(out.data(), dout, sizeof(double) * 6 * nfit, cudaMemcpyDeviceToHost, st));
            STPGPU_CUDA_TRY(cudaMemcpyAsync(its.data(), dit, sizeof(int) * nfit, cudaMemcpyDeviceToHost, st));
            STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
            for (int k = 0; k < nfit; k++) {
                stpgpu_island& o = islands[which[k]];
                for (int q = 0; q < 6; q++)
                    o.leastsq_fit[q] = out[6 * size_t(k) + q];
                constrain(o.leastsq_fit); // fitting.cpp:32-57
                o.fit_iterations = its[k];
            }
        }
    }
}

} // namespace

// ====================================================================== C ABI

extern "C" {

int stpgpu_abi_version(void) { return STPGPU_ABI_VERSION; }

stpgpu_status stpgpu_create(int device, stpgpu_context** out)
{
    if (!out)
        return STPGPU_ERR_INVALID_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return STPGPU_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev)
        return STPGPU_ERR_INVALID_ARG;
    stpgpu_context* c = new stpgpu_context();
    c->device = device;
    stpgpu_status s = guard(c, [&] {
        STPGPU_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        STPGPU_CUDA_TRY(cudaEventCreate(&c->ev0));
        STPGPU_CUDA_TRY(cudaEventCreate(&c->ev1));
    });
    if (s != STPGPU_OK) {
        delete c;
        return s;
    }
    *out = c;
    return STPGPU_OK;
}

stpgpu_status stpgpu_destroy(stpgpu_context* c)
{
    if (!c)
        return STPGPU_OK;
    cudaSetDevice(c->device);
    c->release();
    if (c->pinned)
        cudaFreeHost(c->pinned);
    if (c->batch_host)
        cudaFreeHost(c->batch_host);
    for (auto w : c->wstreams)
        cudaStreamDestroy(w);
    for (auto e : c->wevents)
        cudaEventDestroy(e);
    if (c->fork_ev)
        cudaEventDestroy(c->fork_ev);
    for (auto e : c->tev)
        if (e)
            cudaEventDestroy(e);
    if (c->ev0)
        cudaEventDestroy(c->ev0);
    if (c->ev1)
        cudaEventDestroy(c->ev1);
    for (auto& e : c->pev)
        if (e)
            cudaEventDestroy(e);
    if (c->stream)
        cudaStreamDestroy(c->stream);
    delete c;
    return STPGPU_OK;
}

const char* stpgpu_last_error(const stpgpu_context* c) { return c ? c->err.c_str() : "null context"; }

void* stpgpu_stream(stpgpu_context* c) { return c ? reinterpret_cast<void*>(c->stream) : nullptr; }

stpgpu_status stpgpu_trim(stpgpu_context* c)
{
    return guard(c, [&] { c->release(); });
}

stpgpu_status stpgpu_image_visibilities_ex(stpgpu_context* c, const void* vis, int vis_dtype, const double* weights,
    const double* uvw, int64_t n_vis, const stpgpu_imager_pars* pars, const stpgpu_wproj_pars* wproj,
    const stpgpu_aproj_pars* aproj, int precision, void* image, void* beam, int out_dtype, int device_ptrs,
    stpgpu_imager_info* info)
{
    return guard(c, [&] {
        int image_size = 0;
        ImagerSetup s = setup_from(pars, wproj, aproj, image_size);
        if (n_vis < 0 || (n_vis > 0 && (!vis || !weights || !uvw)) || !image)
            fail(STPGPU_ERR_INVALID_ARG, "null buffer");
        if (vis_dtype != STPGPU_C128 && vis_dtype != STPGPU_C64)
            fail(STPGPU_ERR_INVALID_ARG, "vis_dtype");
        if (out_dtype != STPGPU_F64 && out_dtype != STPGPU_F32)
            fail(STPGPU_ERR_INVALID_ARG, "out_dtype");
        const int vc64 = vis_dtype == STPGPU_C64;
        const size_t vbytes = vc64 ? 8 : 16;
        const void* dv = vis;
        const double* dw = weights;
        const double* duvw = uvw;
        const bool timed = !device_ptrs;
        if (timed)
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
        if (s.ntimesteps > 0 && n_vis > 0 && !s.lha)
            fail(STPGPU_ERR_INVALID_ARG, "A-projection needs the hour angle of every visibility (lha)");
        if (!device_ptrs) {
            dv = to_device<unsigned char>(c, "in_vis", vis, vbytes * size_t(n_vis));
            dw = to_device<double>(c, "in_w", weights, size_t(n_vis));
            duvw = to_device<double>(c, "in_uvw", uvw, 3 * size_t(n_vis));
            if (s.ntimesteps > 0)
                s.lha = to_device<double>(c, "in_lha", s.lha, size_t(n_vis));
        }
        const int64_t npix = int64_t(image_size) * image_size;
        const size_t obytes = out_dtype == STPGPU_F32 ? 4 : 8;
        void* dimg = image;
        void* dbeam = beam;
        if (!device_ptrs) {
            dimg = c->buf<unsigned char>("out_img", obytes * size_t(std::max<int64_t>(npix, 1)));
            dbeam = (s.beam && beam) ? c->buf<unsigned char>("out_beam", obytes * size_t(std::max<int64_t>(npix, 1)))
                                     : nullptr;
        }
        stpgpu_imager_info local {};
        stpgpu_imager_info* inf = info ? info : &local;
        std::memset(inf, 0, sizeof(*inf));
        g_launches = 0;
        const int f32 = out_dtype == STPGPU_F32;
        s.beam = s.beam && beam != nullptr;
        switch (precision) {
        case STPGPU_FP64:
            run_imager<double, 0>(c, s, image_size, pars->gridding_correction, dv, vc64, dw, duvw, n_vis, dimg, dbeam,
                f32, inf, device_ptrs != 0);
            break;
        case STPGPU_FP32:
            run_imager<float, 0>(c, s, image_size, pars->gridding_correction, dv, vc64, dw, duvw, n_vis, dimg, dbeam,
                f32, inf, device_ptrs != 0);
            break;
        case STPGPU_FP32C:
            run_imager<float, 1>(c, s, image_size, pars->gridding_correction, dv, vc64, dw, duvw, n_vis, dimg, dbeam,
                f32, inf, device_ptrs != 0);
            break;
        default:
            fail(STPGPU_ERR_INVALID_ARG, "precision");
        }
        if (!device_ptrs && inf->image_size > 0) {
            STPGPU_CUDA_TRY(cudaMemcpyAsync(image, dimg, obytes * npix, cudaMemcpyDeviceToHost, c->stream));
            if (dbeam)
                STPGPU_CUDA_TRY(cudaMemcpyAsync(beam, dbeam, obytes * npix, cudaMemcpyDeviceToHost, c->stream));
        }
        if (timed)
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (timed) {
            float ms = 0.f;
            STPGPU_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
            inf->device_ms = ms;
        }
        inf->n_launches = g_launches;
    });
}

stpgpu_status stpgpu_image_batch(stpgpu_context* c, const stpgpu_snapshot* snapshots, int32_t n_snapshots,
    int precision, int out_dtype, int device_ptrs, stpgpu_imager_info* infos, stpgpu_batch_info* batch_info)
{
    return guard(c, [&] {
        if (!snapshots || n_snapshots <= 0)
            fail(STPGPU_ERR_INVALID_ARG, "empty batch");
        if (out_dtype != STPGPU_F64 && out_dtype != STPGPU_F32)
            fail(STPGPU_ERR_INVALID_ARG, "out_dtype");
        const int f32 = out_dtype == STPGPU_F32;
        switch (precision) {
        case STPGPU_FP64:
            run_batch<double, 0>(c, snapshots, n_snapshots, precision, f32, device_ptrs, infos, batch_info);
            break;
        case STPGPU_FP32:
            run_batch<float, 0>(c, snapshots, n_snapshots, precision, f32, device_ptrs, infos, batch_info);
            break;
        case STPGPU_FP32C:
            run_batch<float, 1>(c, snapshots, n_snapshots, precision, f32, device_ptrs, infos, batch_info);
            break;
        default:
            fail(STPGPU_ERR_INVALID_ARG, "precision");
        }
    });
}

stpgpu_status stpgpu_model_visibilities(stpgpu_context* c, const double* skymodel, int32_t n_src, const double* uvw,
    int64_t n_vis, const double* vis_in, double* vis_out, int device_ptrs)
{
    return guard(c, [&] {
        if (n_src < 0 || n_vis < 0 || (n_vis > 0 && (!uvw || !vis_out)) || (n_src > 0 && !skymodel))
            fail(STPGPU_ERR_INVALID_ARG, "null buffer or negative size");
        if (n_vis == 0)
            return;
        cudaStream_t st = c->stream;
        const double* dsky = skymodel;
        const double* duvw = uvw;
        const double* dvin = vis_in;
        double* dout = vis_out;
        if (!device_ptrs) {
            dsky = to_device<double>(c, "mv_sky", skymodel, 3 * size_t(n_src));
            duvw = to_device<double>(c, "mv_uvw", uvw, 3 * size_t(n_vis));
            if (vis_in)
                dvin = to_device<double>(c, "mv_in", vis_in, 2 * size_t(n_vis));
            dout = c->buf<double>("mv_out", 2 * size_t(n_vis));
        }
        k_model_vis<<<grid1d(n_vis, VIS_THREADS), VIS_THREADS, 0, st>>>(dsky, n_src, duvw, n_vis, dvin,
            vis_in != nullptr, dout);
        STPGPU_CHECK_LAUNCH();
        if (!device_ptrs)
            STPGPU_CUDA_TRY(cudaMemcpyAsync(vis_out, dout, 2 * sizeof(double) * size_t(n_vis), cudaMemcpyDeviceToHost, st));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(st));
    });
}

stpgpu_status stpgpu_set_timing(stpgpu_context* c, int enable)
{
    return guard(c, [&] {
        if (enable)
            for (auto& e : c->pev)
                if (!e)
                    STPGPU_CUDA_TRY(cudaEventCreate(&e));
        c->timing = enable != 0;
    });
}

stpgpu_status stpgpu_image_visibilities(stpgpu_context* c, const double* vis, const double* weights, const double* uvw,
    int64_t n_vis, const stpgpu_imager_pars* pars, const stpgpu_wproj_pars* wproj, const stpgpu_aproj_pars* aproj,
    double* image, double* beam, stpgpu_imager_info* info)
{
    return stpgpu_image_visibilities_ex(c, vis, STPGPU_C128, weights, uvw, n_vis, pars, wproj, aproj, STPGPU_FP64,
        image, beam, STPGPU_F64, 0, info);
}

stpgpu_status stpgpu_convolve_to_grid(stpgpu_context* c, int kernel_function, double kernel_trunc, int support,
    int image_size, const double* uv, const double* vis, const double* weights, int64_t n_vis, int kernel_exact,
    int oversampling, int shift_uv, int halfplane, int generate_beam, const stpgpu_wproj_pars* wproj, const double* w,
    double cell_size, int analytic_gcf, double* vis_grid, double* sampling_grid, double* sample_grid_total)
{
    return guard(c, [&] {
        if (kernel_function < 0 || kernel_function > 5)
            fail(STPGPU_ERR_INVALID_ARG, "unknown kernel function");
        if (n_vis < 0 || (n_vis > 0 && (!uv || !vis || !weights)) || !vis_grid)
            fail(STPGPU_ERR_INVALID_ARG, "null buffer");
        ImagerSetup s;
        s.kf = kernel_function;
        s.trunc = kernel_trunc;
        s.support = support;
        s.N = image_size;
        s.kernel_exact = kernel_exact;
        s.os = oversampling;
        s.shift_uv = shift_uv;
        s.halfplane = halfplane;
        s.beam = generate_beam && sampling_grid;
        s.analytic = analytic_gcf;
        s.cell_size = cell_size;
        const bool wp = wproj && wproj->num_wplanes > 0;
        if (wp) {
            if (!w)
                fail(STPGPU_ERR_INVALID_ARG, "W-projection needs w");
            if (!(cell_size > 0.0))
                fail(STPGPU_ERR_INVALID_ARG, "W-projection needs cell_size > 0");
            s.nplanes = wproj->num_wplanes;
            s.max_support = wproj->max_wpconv_support;
            s.undersampling = wproj->undersampling_opt;
            s.trunc_perc = wproj->kernel_trunc_perc;
            s.wmedian = wproj->wplanes_median;
            if (wproj->hankel_opt) {
                if (wproj->interp_type < 0 || wproj->interp_type > 2)
                    fail(STPGPU_ERR_INVALID_ARG, "unknown interp_type");
                s.hankel = 1;
                s.proj_slice = wproj->hankel_proj_slice ? 1 : 0;
                s.cubic = wproj->interp_type == 1;
            }
        }
        if (!kernel_exact && !wp && oversampling < 1)
            fail(STPGPU_ERR_INVALID_ARG, "oversampling must be >= 1");
        // uv (n x 2) [+ w] in pixels as an n x 3 device array
        double* duv = c->buf<double>("in_uv", 3 * size_t(std::max<int64_t>(n_vis, 1)));
        if (n_vis) {
            STPGPU_CUDA_TRY(cudaMemcpyAsync(duv, uv, sizeof(double) * 2 * n_vis, cudaMemcpyHostToDevice, c->stream));
            if (wp)
                STPGPU_CUDA_TRY(
                    cudaMemcpyAsync(duv + 2 * n_vis, w, sizeof(double) * n_vis, cudaMemcpyHostToDevice, c->stream));
        }
        const double* dvis = to_device<double>(c, "in_vis", vis, 2 * size_t(n_vis));
        const double* dw = to_device<double>(c, "in_w", weights, size_t(n_vis));
        c->drop_single(); // this call reuses the imager's buffers
        GridOut g = run_gridder<double, 0>(c, s, dvis, 0, dw, duv, 1, n_vis);
        ScalarsBack sb = read_back(c, g);
        if (sb.err & 4u) { // redo with the 64-bit |w| sort
            s.full_wsort = 1;
            g = run_gridder<double, 0>(c, s, dvis, 0, dw, duv, 1, n_vis);
            sb = read_back(c, g);
        }
        const size_t cells = size_t(g.image_rows) * size_t(image_size);
        STPGPU_CUDA_TRY(cudaMemcpyAsync(vis_grid, g.grid, sizeof(double2) * cells, cudaMemcpyDeviceToHost, c->stream));
        if (s.beam)
            STPGPU_CUDA_TRY(
                cudaMemcpyAsync(sampling_grid, g.beam, sizeof(double2) * cells, cudaMemcpyDeviceToHost, c->stream));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (sample_grid_total)
            *sample_grid_total = sb.total;
    });
}

stpgpu_status stpgpu_source_find_ex(stpgpu_context* c, const void* image, int image_dtype, int32_t rows, int32_t cols,
    const stpgpu_sf_pars* pars, int32_t* label_map, int device_ptrs, stpgpu_island* islands, int32_t capacity,
    int32_t* n_islands, stpgpu_sf_info* info)
{
    return guard(c, [&] {
        if (!image || !pars || !n_islands)
            fail(STPGPU_ERR_INVALID_ARG, "null argument");
        if (image_dtype != STPGPU_F64 && image_dtype != STPGPU_F32)
            fail(STPGPU_ERR_INVALID_ARG, "image_dtype");
        const int64_t n = int64_t(rows) * cols;
        const size_t eb = image_dtype == STPGPU_F32 ? 4 : 8;
        if (!device_ptrs)
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
        const void* dimg = image;
        if (!device_ptrs && n > 0)
            dimg = to_device<unsigned char>(c, "sf_in", image, eb * size_t(n));
        int32_t* dl = device_ptrs ? label_map : nullptr;
        std::vector<stpgpu_island> isl;
        stpgpu_sf_info local {};
        stpgpu_sf_info* inf = info ? info : &local;
        std::memset(inf, 0, sizeof(*inf));
        const bool want = label_map != nullptr;
        if (image_dtype == STPGPU_F32)
            run_source_find<float>(c, reinterpret_cast<const float*>(dimg), rows, cols, *pars, dl, want, isl, *inf);
        else
            run_source_find<double>(c, reinterpret_cast<const double*>(dimg), rows, cols, *pars, dl, want, isl, *inf);
        if (!device_ptrs && label_map) {
            const int32_t* src = c->buf<int32_t>("ccl_L", n);
            STPGPU_CUDA_TRY(cudaMemcpyAsync(label_map, src, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c->stream));
        }
        if (!device_ptrs)
            STPGPU_CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
        STPGPU_CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (!device_ptrs) {
            float ms = 0.f;
            STPGPU_CUDA_TRY(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
            inf->device_ms = ms;
        }
        *n_islands = int32_t(isl.size());
        if (int32_t(isl.size()) > capacity)
            fail(STPGPU_ERR_CAPACITY, "island buffer too small: need " + std::to_string(isl.size()));
        if (!isl.empty())
            std::memcpy(islands, isl.data(), sizeof(stpgpu_island) * isl.size());
    });
}

stpgpu_status stpgpu_source_find(stpgpu_context* c, const double* image, int32_t rows, int32_t cols,
    const stpgpu_sf_pars* pars, int32_t* label_map, stpgpu_island* islands, int32_t capacity, int32_t* n_islands,
    stpgpu_sf_info* info)
{
    return stpgpu_source_find_ex(c, image, STPGPU_F64, rows, cols, pars, label_map, 0, islands, capacity, n_islands,
        info);
}

} // extern "C"

// ------------------------------------------------------------------ serving

namespace {

struct ServerJob {
    int64_t ticket = 0;
    stpgpu_request req {};
    stpgpu_result res {};
    bool done = false;
};

// Device working set of one request (inputs, items, tile lists, W-planes and
// W-kernel tables, grid, FFT output, image, source-finder arrays), bytes.
int64_t request_bytes(const ImagerSetup& s, int image_size, int64_t n, int vis_c64, int precision, int find_sources,
    int correction)
{
    const int64_t rb = precision == STPGPU_FP64 ? 8 : 4;
    const int64_t N = s.N, rows = N / 2 + 1;
    const int conv = s.nplanes > 0 ? s.max_support : s.support;
    int64_t b = n * ((vis_c64 ? 8 : 16) + 8 + 24) + n * (rb == 8 ? 48 : 32); // items: 48 / 32 B records
    const int64_t per_dim = ceil_div(2 * conv, 16) + 2;
    b += std::max<int64_t>(n, 1) * 2 * per_dim * per_dim * 4; // tile-list capacity
    b += std::max<int64_t>(n, 1) * 2 * kRankSlots * 4;         // list slots kept by the count pass
    if (s.nplanes > 0) {
        b += n * (rb == 8 ? 48 : 32); // items in |w| order
        const int64_t os = std::max(1, (s.os >> 1) << 1), cs = (os / 2) * 2 + 1, K = 2 * conv + 1;
        const int64_t lh = conv * os + os / 2 + 1;
        b += n * 41;                                                  // |w| sort, planes
        b += int64_t(s.nplanes) * (cs * cs * K * K * 2 * rb + lh * lh * 16 + 64 * 64 * 16);
    }
    b += rows * N * 2 * rb + N * N * rb + int64_t(image_size) * image_size * rb;
    if (precision == STPGPU_FP32C && wide_fft_needed(s, image_size, correction))
        b += rows * N * 2 * rb + N * N * rb; // double-precision grid and c2r output
    if (find_sources) // classes, parents, ranks, labels, foreground list; at worst list arrays (20 B) for every
                      // pixel and per-label arrays (160 B) for every second pixel
        b += int64_t(image_size) * image_size * (1 + 4 + 4 + 4 + 4 + 20 + 80 + 2) + (int64_t(8) << 20); // + clip lists
    return b + (int64_t(8) << 20);
}

// One request on one slot context (host buffers in and out).
template <typename R, int COMP>
void serve_request(stpgpu_context* c, const stpgpu_request& r, stpgpu_result& res)
{
    int image_size = 0;
    ImagerSetup s = setup_from(&r.pars, &r.wproj, nullptr, image_size);
    s.beam = 0;
    const int c64 = r.vis_dtype == STPGPU_C64;
    const int f32 = r.out_dtype == STPGPU_F32;
    const int64_t n = r.n_vis;
    const void* dv = to_device<unsigned char>(c, "in_vis", r.vis, (c64 ? 8 : 16) * size_t(n));
    const double* dw = to_device<double>(c, "in_w", r.weights, size_t(n));
    const double* duvw = to_device<double>(c, "in_uvw", r.uvw, 3 * size_t(n));
    const int64_t npix = int64_t(image_size) * image_size;
    const size_t ob = f32 ? 4 : 8;
    void* dimg = c->buf<unsigned char>("srv_img", ob * size_t(std::max<int64_t>(npix, 1)));
    const auto t_in = std::chrono::steady_clock::now();
    run_imager<R, COMP>(c, s, image_size, r.pars.gridding_correction, dv, c64, dw, duvw, n, dimg, nullptr, f32,
        &res.imager);
    const auto t_img = std::chrono::steady_clock::now();
    if (res.imager.image_size > 0) {
        if (r.image)
            STPGPU_CUDA_TRY(cudaMemcpyAsync(r.image, dimg, ob * npix, cudaMemcpyDeviceToHost, c->stream));
        if (r.find_sources) {
            std::vector<stpgpu_island> isl;
            if (f32)
                run_source_find<float>(c, reinterpret_cast<const float*>(dimg), image_size, image_size, r.sf, nullptr,
                    r.label_map != nullptr, isl, res.sf);
            else
                run_source_find<double>(c, reinterpret_cast<const double*>(dimg), image_size, image_size, r.sf,
                    nullptr, r.label_map != nullptr, isl, res.sf);
            if (r.label_map)
                STPGPU_CUDA_TRY(cudaMemcpyAsync(r.label_map, c->buf<int32_t>("ccl_L", npix), sizeof(int32_t) * npix,
                    cudaMemcpyDeviceToHost, c->stream));
            res.n_islands = int32_t(isl.size());
            if (int32_t(isl.size()) > r.island_capacity)
                fail(STPGPU_ERR_CAPACITY, "island buffer too small: need " + std::to_string(isl.size()));
            if (!isl.empty())
                std::memcpy(r.islands, isl.data(), sizeof(stpgpu_island) * isl.size());
        }
    }
    STPGPU_CUDA_TRY(cudaStreamSynchronize(c->stream));
    // STPGPU_LOG_SLOW=<ms>: host-side phase times of requests slower than that
    static const char* slow = std::getenv("STPGPU_LOG_SLOW");
    if (slow) {
        const auto t_end = std::chrono::steady_clock::now();
        auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
        if (ms(t_in, t_end) > std::atof(slow))
            std::fprintf(stderr, "stpgpu slow request: N=%d n_vis=%lld imager %.3f ms, source finder %.3f ms\n",
                image_size, (long long)n, ms(t_in, t_img), ms(t_img, t_end));
    }
}

} // namespace

struct stpgpu_server {
    stpgpu_server_pars pars {};
    std::vector<stpgpu_context*> slots;
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ServerJob*> queue;
    std::unordered_map<int64_t, std::unique_ptr<ServerJob>> jobs;
    int64_t next_ticket = 1;
    int64_t inflight = 0, inflight_bytes = 0;
    bool stop = false;
    int paused = 0; // stpgpu_server_prepare holds the slots: no admission
    std::chrono::steady_clock::time_point t0;
    std::vector<double> latency_ms;
    double first_submit = -1.0, last_done = 0.0;
    stpgpu_server_stats st {};

    double now_ms() const
    {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }

    void worker(int k)
    {
        stpgpu_context* c = slots[k];
        cudaSetDevice(c->device);
        for (;;) {
            ServerJob* job = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                // first-in first-out: the head starts once its working set fits
                auto admissible = [&] {
                    return !paused && !queue.empty()
                        && inflight_bytes + queue.front()->res.est_bytes <= pars.hbm_budget_bytes;
                };
                cv_work.wait(lk, [&] { return stop || admissible(); });
                if (queue.empty() && stop)
                    return;
                if (!admissible())
                    continue;
                job = queue.front();
                queue.pop_front();
                inflight++;
                inflight_bytes += job->res.est_bytes;
                st.peak_in_flight = std::max(st.peak_in_flight, inflight);
                st.peak_admitted_bytes = std::max(st.peak_admitted_bytes, inflight_bytes);
                job->res.admit_ms = now_ms();
            }
            const stpgpu_status status = guard(c, [&] {
                g_launches = 0;
                switch (pars.precision) {
                case STPGPU_FP64:
                    serve_request<double, 0>(c, job->req, job->res);
                    break;
                case STPGPU_FP32:
                    serve_request<float, 0>(c, job->req, job->res);
                    break;
                default:
                    serve_request<float, 1>(c, job->req, job->res);
                    break;
                }
            });
            {
                std::lock_guard<std::mutex> lk(mu);
                job->res.status = status;
                if (status != STPGPU_OK)
                    std::snprintf(job->res.error, sizeof(job->res.error), "%s", c->err.c_str());
                job->res.done_ms = now_ms();
                job->done = true;
                inflight--;
                inflight_bytes -= job->res.est_bytes;
                if (status == STPGPU_OK) {
                    st.completed++;
                    latency_ms.push_back(job->res.done_ms - job->res.submit_ms);
                    last_done = std::max(last_done, job->res.done_ms);
                } else {
                    st.failed++;
                }
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }
};

extern "C" {

stpgpu_status stpgpu_server_create(const stpgpu_server_pars* pars, stpgpu_server** out)
{
    if (!pars || !out || pars->slots < 1 || pars->hbm_budget_bytes <= 0)
        return STPGPU_ERR_INVALID_ARG;
    if (pars->precision < STPGPU_FP64 || pars->precision > STPGPU_FP32C)
        return STPGPU_ERR_INVALID_ARG;
    *out = nullptr;
    auto* sv = new stpgpu_server();
    sv->pars = *pars;
    sv->t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < pars->slots; k++) {
        stpgpu_context* c = nullptr;
        const stpgpu_status s = stpgpu_create(pars->device, &c);
        if (s != STPGPU_OK) {
            for (auto x : sv->slots)
                stpgpu_destroy(x);
            delete sv;
            return s;
        }
        if (!sv->slots.empty())
            c->tunes = sv->slots[0]->tunes; // a size class is tuned once for all slots
        sv->slots.push_back(c);
    }
    for (int k = 0; k < pars->slots; k++)
        sv->workers.emplace_back([sv, k] { sv->worker(k); });
    *out = sv;
    return STPGPU_OK;
}

stpgpu_status stpgpu_server_destroy(stpgpu_server* sv)
{
    if (!sv)
        return STPGPU_OK;
    {
        std::unique_lock<std::mutex> lk(sv->mu);
        sv->cv_done.wait(lk, [&] { return sv->queue.empty() && sv->inflight == 0; });
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    for (auto& t : sv->workers)
        t.join();
    for (auto c : sv->slots)
        stpgpu_destroy(c);
    delete sv;
    return STPGPU_OK;
}

namespace {

// Parameter checks of a request and its working-set estimate.
stpgpu_status check_request(const stpgpu_server* sv, const stpgpu_request* r, int64_t& est)
{
    est = 0;
    try {
        int image_size = 0;
        ImagerSetup s = setup_from(&r->pars, &r->wproj, nullptr, image_size);
        if (r->pars.generate_beam)
            return STPGPU_ERR_UNSUPPORTED;
        if (image_size <= 0 || image_size > s.N || (image_size % 2) != 0)
            return STPGPU_ERR_INVALID_ARG;
        if (r->n_vis < 0 || (r->n_vis > 0 && (!r->vis || !r->weights || !r->uvw)) || (!r->image && !r->find_sources))
            return STPGPU_ERR_INVALID_ARG;
        if ((r->vis_dtype != STPGPU_C128 && r->vis_dtype != STPGPU_C64)
            || (r->out_dtype != STPGPU_F64 && r->out_dtype != STPGPU_F32))
            return STPGPU_ERR_INVALID_ARG;
        if (r->find_sources && (r->island_capacity < 0 || (r->island_capacity > 0 && !r->islands)))
            return STPGPU_ERR_INVALID_ARG;
        est = request_bytes(s, image_size, r->n_vis, r->vis_dtype == STPGPU_C64, sv->pars.precision, r->find_sources,
            r->pars.gridding_correction);
    } catch (const Error& e) {
        return e.status;
    }
    if (est > sv->pars.hbm_budget_bytes)
        return STPGPU_ERR_OOM;
    return STPGPU_OK;
}

} // namespace

stpgpu_status stpgpu_server_submit(stpgpu_server* sv, const stpgpu_request* r, int64_t* ticket)
{
    if (!sv || !r || !ticket)
        return STPGPU_ERR_INVALID_ARG;
    int64_t est = 0;
    if (const stpgpu_status bad = check_request(sv, r, est))
        return bad;
    auto job = std::make_unique<ServerJob>();
    job->req = *r;
    job->res.est_bytes = est;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        job->ticket = sv->next_ticket++;
        job->res.submit_ms = sv->now_ms();
        if (sv->first_submit < 0)
            sv->first_submit = job->res.submit_ms;
        sv->st.submitted++;
        *ticket = job->ticket;
        sv->queue.push_back(job.get());
        sv->jobs[job->ticket] = std::move(job);
    }
    sv->cv_work.notify_all();
    return STPGPU_OK;
}

stpgpu_status stpgpu_server_prepare(stpgpu_server* sv, const stpgpu_request* r, stpgpu_result* out)
{
    if (!sv || !r)
        return STPGPU_ERR_INVALID_ARG;
    stpgpu_result res {};
    if (const stpgpu_status bad = check_request(sv, r, res.est_bytes))
        return bad;
    {
        // hold admission and let the requests in flight finish: the slots'
        // contexts are then free for this thread
        std::unique_lock<std::mutex> lk(sv->mu);
        sv->paused++;
        sv->cv_done.wait(lk, [&] { return sv->inflight == 0; });
    }
    stpgpu_status status = STPGPU_OK;
    for (stpgpu_context* c : sv->slots) {
        cudaSetDevice(c->device);
        res = stpgpu_result {};
        status = guard(c, [&] {
            switch (sv->pars.precision) {
            case STPGPU_FP64:
                serve_request<double, 0>(c, *r, res);
                break;
            case STPGPU_FP32:
                serve_request<float, 0>(c, *r, res);
                break;
            default:
                serve_request<float, 1>(c, *r, res);
                break;
            }
        });
        if (status != STPGPU_OK) {
            std::snprintf(res.error, sizeof(res.error), "%s", c->err.c_str());
            break;
        }
    }
    res.status = status;
    if (out)
        *out = res;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->paused--;
    }
    sv->cv_work.notify_all();
    return status;
}

stpgpu_status stpgpu_server_wait(stpgpu_server* sv, int64_t ticket, double timeout_s, stpgpu_result* out)
{
    if (!sv)
        return STPGPU_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(ticket);
    if (it == sv->jobs.end())
        return STPGPU_ERR_INVALID_ARG;
    ServerJob* job = it->second.get();
    if (timeout_s < 0)
        sv->cv_done.wait(lk, [&] { return job->done; });
    else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return job->done; }))
        return STPGPU_ERR_TIMEOUT;
    if (out)
        *out = job->res;
    const stpgpu_status s = stpgpu_status(job->res.status);
    sv->jobs.erase(it);
    return s;
}

stpgpu_status stpgpu_server_stats_get(stpgpu_server* sv, stpgpu_server_stats* out)
{
    if (!sv || !out)
        return STPGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(sv->mu);
    stpgpu_server_stats s = sv->st;
    s.in_flight = sv->inflight;
    s.queued = int64_t(sv->queue.size());
    std::vector<double> l = sv->latency_ms;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto pct = [&](double q) {
            const double pos = q * double(l.size() - 1);
            const size_t i = size_t(pos);
            const double f = pos - double(i);
            return i + 1 < l.size() ? l[i] * (1.0 - f) + l[i + 1] * f : l[i];
        };
        s.p50_ms = pct(0.50);
        s.p99_ms = pct(0.99);
        double sum = 0.0;
        for (double v : l)
            sum += v;
        s.mean_ms = sum / double(l.size());
        const double span = sv->last_done - sv->first_submit;
        s.throughput_rps = span > 0 ? double(s.completed) / (span / 1e3) : 0.0;
    }
    *out = s;
    return STPGPU_OK;
}

} // extern "C"

// ------------------------------------------------------- allocation-free labelling
//
// stpgpu_label_noalloc runs the connected-component labeller (k_ccl_* above)
// with its working arrays in one file-scope device array instead of
// context-owned buffers.  It exists for callers that must not allocate:
//  * a real-time detection stage that runs between the imaging launches of a
//    stream-ordered pipeline: cudaMalloc/cudaFree synchronise the whole device
//    and would stall the imaging streams that share it, breaking the snapshot
//    cadence;
//  * a process whose device memory is already owned by another allocator (a
//    caching allocator or a memory pool that reserved the free HBM up front),
//    where an allocation by this library could fail with out-of-memory in the
//    middle of a run;
// neither can create a stpgpu_context, which allocates its buffers, stream and
// events.  The call makes no cudaMalloc, cudaFree or allocating library call;
// host-side it uses no heap either (no exceptions, strings or containers).
//
// Scratch layout for n = rows * cols pixels (byte offsets, 256-aligned):
//   cls  nchunks * CCL_CHUNK bytes   pixel class (0 background, 1 positive,
//                       2 negative), background padding past n
//   P    n uint32       union-find parents
//   R    n uint32       final label number of each root
//   misc 8 uint32       row totals and the union-find step-bound flag; the
//                       flag MUST start at zero, so every call clears misc
//                       before the first kernel
//   cnt, off            3 * (nchunks + 1) uint32 each: positive roots,
//                       negative roots and foreground keys per chunk of
//                       CCL_CHUNK keys, and their exclusive scans
// Everything except misc is fully written before it is read in each call.
// The array is shared by every call on a device: two calls whose kernels
// overlap on the GPU (different streams, or different host threads) race on
// it and give wrong labels.  The first call on a device resolves the array's
// device address (cudaGetSymbolAddress, that device current) and caches it;
// that first call should come before any stream capture.

namespace stpgpu {

constexpr size_t noalloc_align(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t noalloc_chunks(size_t n) { return (n + CCL_CHUNK - 1) / CCL_CHUNK; }
constexpr size_t noalloc_bytes(size_t n)
{
    return noalloc_align(noalloc_chunks(n) * CCL_CHUNK) + 2 * noalloc_align(4 * n) + 256
        + 2 * noalloc_align(12 * (noalloc_chunks(n) + 1));
}
constexpr size_t kNoallocScratchBytes = noalloc_bytes(STPGPU_NOALLOC_MAX_PIXELS);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kNoallocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_ptr[kNoallocMaxDevices] = {};

static stpgpu_status noalloc_msg(char* buf, size_t len, stpgpu_status s, const char* what, cudaError_t e)
{
    if (buf && len)
        std::snprintf(buf, len, "%s%s%s", what, e == cudaSuccess ? "" : ": ",
            e == cudaSuccess ? "" : cudaGetErrorString(e));
    return s;
}

template <typename T>
static cudaError_t noalloc_label_run(unsigned char* base, cudaStream_t st, const T* img, int rows, int cols,
    double tp, double tn, int findneg, int conn4, int slice, int32_t* L, uint32_t* h)
{
    const int64_t n = int64_t(rows) * cols;
    const size_t nch = noalloc_chunks(size_t(n));
    size_t o = 0;
    CclBufs b;
    b.cls = base + o;
    o += noalloc_align(nch * CCL_CHUNK);
    b.P = reinterpret_cast<uint32_t*>(base + o);
    o += noalloc_align(4 * size_t(n));
    b.R = reinterpret_cast<uint32_t*>(base + o);
    o += noalloc_align(4 * size_t(n));
    b.misc = reinterpret_cast<uint32_t*>(base + o);
    o += 256;
    b.cnt = reinterpret_cast<uint32_t*>(base + o);
    o += noalloc_align(12 * (nch + 1));
    b.off = reinterpret_cast<uint32_t*>(base + o);
    b.fgl = nullptr;
    b.L = L;
    cudaError_t e = cudaMemsetAsync(b.misc, 0, 8 * sizeof(uint32_t), st);
    if (e != cudaSuccess)
        return e;
    const CclGeom geom { rows, cols, rows / 2, cols / 2 };
    if ((e = ccl_enqueue<T>(st, img, geom, nullptr, tp, tn, findneg, conn4, slice, b)) != cudaSuccess)
        return e;
    // label counts and the step-bound flag, read back into host stack memory
    if ((e = cudaMemcpyAsync(h, b.misc, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(st);
}

} // namespace stpgpu

extern "C" stpgpu_status stpgpu_label_noalloc(int device, void* stream, const void* image, int image_dtype,
    int32_t rows, int32_t cols, double analysis_thresh_pos, double analysis_thresh_neg, int find_negative_sources,
    int ccl_4connectivity, int ccl_slice_cols, int32_t* label_map, int32_t* n_labels_pos, int32_t* n_labels_neg,
    char* err_msg, size_t err_msg_len)
{
    using namespace stpgpu;
    if (err_msg && err_msg_len)
        err_msg[0] = '\0';
    if (!image || !label_map)
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_INVALID_ARG, "null image or label_map", cudaSuccess);
    if (image_dtype != STPGPU_F64 && image_dtype != STPGPU_F32)
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_INVALID_ARG, "image_dtype", cudaSuccess);
    if (rows <= 0 || cols <= 0 || (rows % 2) || (cols % 2) || rows > 65536 || cols > 65536)
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_INVALID_ARG,
            "image dimensions must be positive, even and at most 65536 (ccl.h:116-119)", cudaSuccess);
    if (int64_t(rows) * cols > int64_t(STPGPU_NOALLOC_MAX_PIXELS)) {
        if (err_msg && err_msg_len)
            std::snprintf(err_msg, err_msg_len,
                "image of %lld pixels exceeds the allocation-free labeller's maximum of %lld pixels",
                (long long)(int64_t(rows) * cols), (long long)STPGPU_NOALLOC_MAX_PIXELS);
        return STPGPU_ERR_INVALID_ARG;
    }
    if (device < 0 || device >= kNoallocMaxDevices)
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_INVALID_ARG, "device ordinal", cudaSuccess);
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess)
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_NO_DEVICE, "cudaGetDevice", e);
    if ((e = cudaSetDevice(device)) != cudaSuccess)
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_NO_DEVICE, "cudaSetDevice", e);
    unsigned char* base = nullptr;
    {
        // set-up, once per device, with that device current
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[device]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                cudaSetDevice(prev);
                return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_CUDA, "cudaGetSymbolAddress(scratch)", e);
            }
            g_noalloc_ptr[device] = static_cast<unsigned char*>(p);
        }
        base = g_noalloc_ptr[device];
    }
    const int slice = ccl_slice_cols > 0 ? ccl_slice_cols : std::max(2, cols / 8);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t h[4] = { 0, 0, 0, 0 }; // positive labels, negative labels, foreground keys, step-bound flag
    if (image_dtype == STPGPU_F32)
        e = noalloc_label_run<float>(base, st, static_cast<const float*>(image), rows, cols, analysis_thresh_pos,
            analysis_thresh_neg, find_negative_sources, ccl_4connectivity, slice, label_map, h);
    else
        e = noalloc_label_run<double>(base, st, static_cast<const double*>(image), rows, cols, analysis_thresh_pos,
            analysis_thresh_neg, find_negative_sources, ccl_4connectivity, slice, label_map, h);
    cudaSetDevice(prev);
    if (e != cudaSuccess)
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_CUDA, "labelling", e);
    if (h[3])
        return noalloc_msg(err_msg, err_msg_len, STPGPU_ERR_DEVICE, "labeler gave up (union-find step bound)",
            cudaSuccess);
    if (n_labels_pos)
        *n_labels_pos = int32_t(h[0]);
    if (n_labels_neg)
        *n_labels_neg = int32_t(h[1]);
    return STPGPU_OK;
}
