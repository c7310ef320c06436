// C ABI of libgt (include/gt.h): argument checking, host<->device staging, error capture.
//
// Every entry point runs its body inside guarded(): CUDA errors and allocation failures become a
// gt_status plus a message on the context, never an exit() (the reference's CUDA entry exits on a
// launch error, shmem/grav_cuda.cu:239-243).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "gt_internal.cuh"

namespace gt {

void set_error(gt_context* ctx, int status, const std::string& msg) {
    if (ctx) ctx->last_error = std::string(gt_status_string(status)) + ": " + msg;
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Fail{e == cudaErrorMemoryAllocation ? GT_ERR_NOMEM : GT_ERR_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(e)};
    }
}

void check_launch(gt_context* ctx, const char* what) {
    ++ctx->launches;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Fail{GT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}

void* scratch(gt_context* ctx, Slot s, size_t bytes) {
    if ((int)ctx->scratch.size() < kSlotCount) ctx->scratch.resize(kSlotCount);
    DevBuf& b = ctx->scratch[s];
    bytes = std::max<size_t>(bytes, 4096);
    if (b.bytes >= bytes) return b.ptr;
    if (b.ptr) {
        // a smaller buffer may still be read by queued work, or written by a queued upload on the
        // copy stream: wait for both streams before freeing
        cudaStreamSynchronize(ctx->stream);
        if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
        cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    const size_t want = bytes + bytes / 8;
    const cudaError_t e = cudaMalloc(&b.ptr, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.ptr = nullptr;
        throw Fail{GT_ERR_NOMEM, "workspace allocation of " + std::to_string(want) + " bytes failed"};
    }
    b.bytes = want;
    return b.ptr;
}

void ensure_copy_stream(gt_context* ctx) {
    if (ctx->copy_stream) return;
    // the events first: the stream marks the set as complete
    auto make = [](cudaEvent_t& e) {
        if (!e) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    };
    for (cudaEvent_t& e : ctx->chunk_ev) make(e);
    for (cudaEvent_t& e : ctx->up_ev) make(e);
    for (cudaEvent_t& e : ctx->down_ev) make(e);
    make(ctx->copy_done);
    make(ctx->main_ev);
    make(ctx->walk2_start);
    make(ctx->walk2_done);
    if (!ctx->walk2) {
        cudaStream_t w = nullptr;
        check_cuda(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking), "cudaStreamCreate");
        ctx->walk2 = w;
    }
    cudaStream_t s = nullptr;
    check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    ctx->copy_stream = s;
}

void* host_stage(gt_context* ctx, size_t bytes) {
    if (ctx->stage_bytes >= bytes) return ctx->stage;
    if (ctx->stage) {
        // queued copies may still use the smaller buffer
        cudaStreamSynchronize(ctx->stream);
        if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
        cudaFreeHost(ctx->stage);
        ctx->stage = nullptr;
        ctx->stage_bytes = 0;
    }
    const size_t want = bytes + bytes / 8;
    void* p = nullptr;
    if (cudaHostAlloc(&p, want, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        throw Fail{GT_ERR_NOMEM, "pinned staging allocation of " + std::to_string(want) + " bytes failed"};
    }
    ctx->stage = p;
    ctx->stage_bytes = want;
    return p;
}

}  // namespace gt

using namespace gt;

namespace {

// A failed call returns only once the second compute stream and the copy stream have drained: no
// upload from, or download into, the caller's host arrays is left running after the error is
// reported.
void drain_copies(gt_context* ctx) {
    if (ctx && ctx->walk2 && cudaStreamSynchronize(ctx->walk2) != cudaSuccess) cudaGetLastError();
    if (ctx && ctx->copy_stream && cudaStreamSynchronize(ctx->copy_stream) != cudaSuccess) cudaGetLastError();
}

template <typename F>
int guarded(gt_context* ctx, F&& body) {
    try {
        body();
        if (ctx) ctx->last_error.clear();
        return GT_OK;
    } catch (const Fail& f) {
        drain_copies(ctx);
        set_error(ctx, f.status, f.msg);
        return f.status;
    } catch (const std::bad_alloc&) {
        drain_copies(ctx);
        set_error(ctx, GT_ERR_NOMEM, "host allocation failed");
        return GT_ERR_NOMEM;
    } catch (...) {
        drain_copies(ctx);
        set_error(ctx, GT_ERR_CUDA, "unexpected exception");
        return GT_ERR_CUDA;
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) check_cuda(cudaSetDevice(dev), "cudaSetDevice");
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Device view of an input array: the pointer itself for GT_MEM_DEVICE, else a staged copy.
template <typename T>
const T* stage_in(gt_context* ctx, Slot s, const T* p, int64_t n, int mem) {
    if (!p) return nullptr;
    if (mem == GT_MEM_DEVICE) return p;
    T* d = (T*)scratch(ctx, s, (size_t)std::max<int64_t>(n, 1) * sizeof(T));
    if (n > 0)
        check_cuda(cudaMemcpyAsync(d, p, (size_t)n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream), "H2D");
    return d;
}

template <typename T>
T* out_buf(gt_context* ctx, Slot s, T* p, int64_t n, int mem) {
    if (!p) return nullptr;
    if (mem == GT_MEM_DEVICE) return p;
    return (T*)scratch(ctx, s, (size_t)std::max<int64_t>(n, 1) * sizeof(T));
}

template <typename T>
void copy_out(gt_context* ctx, T* host, const T* dev, int64_t n, int mem) {
    if (!host || mem == GT_MEM_DEVICE || n <= 0) return;
    check_cuda(cudaMemcpyAsync(host, dev, (size_t)n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
}

void check_mem(int mem) {
    if (mem != GT_MEM_HOST && mem != GT_MEM_DEVICE) throw Fail{GT_ERR_INVALID, "mem must be GT_MEM_HOST or GT_MEM_DEVICE"};
}

void free_tree_arrays(gt_tree* t) {
    void* ptrs[] = {t->src, t->ssoft, t->smass, t->order, t->rank, t->leaf_of, t->sleaf, t->skey,
                    t->nodes, t->parent, t->next, t->level, t->size, t->delta, t->nsoft, t->gc,
                    t->nq2, t->sys_off_dev, t->in_off_dev, t->geom_dev, t->svel, t->nvel, t->vcom, t->vmax,
                    t->m0, t->c0, t->dp, t->dq, t->dmass, t->xpad, t->stype, t->szeta, t->nsink,
                    t->snode, t->hmax};
    // tree arrays came from the stream-ordered pool: hand them back to it (callers have synchronised)
    for (void* p : ptrs)
        if (p) cudaFreeAsync(p, 0);
    for (auto& c : t->group_cache) {
        if (c.groups) {
            if (c.pooled) cudaFreeAsync(c.groups, 0);
            else cudaFree(c.groups);
        }
        if (c.roots) cudaFree(c.roots);
    }
    t->group_cache.clear();
}

void finish(gt_context* ctx, bool sync) {
    if (sync) check_cuda(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
}

void record_walk_time(gt_context* ctx) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->stats.walk_ms = ms;
    cudaGetLastError();
}

void walk_common(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
                 const double* aold, double theta, double G, int group_mode, int group_param,
                 bool leaf_accept, const gt_walk_options* opt, int mem, double* ax, double* ay,
                 double* az, double* phi, WalkBuffers* bufs = nullptr, bool capture = false,
                 double* tidal = nullptr, double* jerk = nullptr) {
    if (!ctx || !tree) throw Fail{GT_ERR_INVALID, "null context or tree"};
    check_mem(mem);
    if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
    if (n_targets < 0) throw Fail{GT_ERR_INVALID, "n_targets < 0"};
    gt_walk_options o;
    gt_walk_options_default(&o);
    if (opt) o = *opt;
    if (o.mac != GT_MAC_PLAIN && o.mac != GT_MAC_LEARNED && o.mac != GT_MAC_NODE)
        throw Fail{GT_ERR_INVALID, "unknown mac"};
    const bool learned = o.mac == GT_MAC_LEARNED || o.mac == GT_MAC_NODE;
    if (learned && !o.mac_model) throw Fail{GT_ERR_INVALID, "a learned criterion needs gt_walk_options.mac_model"};
    if (learned && !leaf_accept)
        throw Fail{GT_ERR_UNSUPPORTED, "the learned criterion applies to the grouped walk"};
    if (o.mac == GT_MAC_NODE)
        for (int i = 0; i < GT_MAC_FEATURES; ++i)
            if (!((GT_MAC_NODE_FEATURES >> i) & 1u) && o.mac_model[GT_MAC_FEATURES + i] != 0.0f)
                throw Fail{GT_ERR_INVALID, "GT_MAC_NODE needs a model that reads node features only"};
    if (o.dtype_out_f32 != 0) throw Fail{GT_ERR_INVALID, "dtype_out_f32 is reserved"};
    if (!(o.sink_direct_radius >= 0.0) || !std::isfinite(o.sink_direct_radius))
        throw Fail{GT_ERR_INVALID, "sink_direct_radius must be finite and >= 0"};
    if (o.out_order == GT_OUT_ORIGINAL && targets) throw Fail{GT_ERR_INVALID, "GT_OUT_ORIGINAL needs targets == NULL"};
    DeviceGuard dg(ctx->device);
    const bool all = targets == nullptr;
    const int64_t nt = all ? tree->n_live : n_targets;
    const int64_t nout = (all && o.out_order == GT_OUT_ORIGINAL) ? tree->n : nt;
    if (!all && nt > 0 && !targets) throw Fail{GT_ERR_INVALID, "targets is null"};
    // Target indices are range-checked on the device as the walk groups them (an index at or
    // beyond the particle count is never dereferenced); a synchronising call reports it below.
    WalkRequest rq;
    rq.targets = all ? nullptr : stage_in(ctx, kSlotIn0, targets, nt, mem);
    rq.n_targets = nt;
    if (mem == GT_MEM_HOST && aold && nt > 0 && !capture) {
        // the walk uploads it: per chunk, ahead of each chunk, when it splits the groups
        rq.aold = (const double*)scratch(ctx, kSlotIn1, (size_t)nt * sizeof(double));
        rq.host_aold = aold;
    } else {
        rq.aold = stage_in(ctx, kSlotIn1, aold, nt, mem);
    }
    rq.theta = theta;
    rq.G = G;
    rq.group_mode = group_mode;
    rq.group_param = group_param;
    rq.leaf_accept = leaf_accept;
    rq.want_acc = ax != nullptr;
    rq.want_phi = phi != nullptr;
    rq.out_original = all && o.out_order == GT_OUT_ORIGINAL;
    rq.mac = o.mac;
    if (learned) {
        if (bufs) {
            // a plan keeps its own device copy, made before capture
            if (!bufs->model) {
                check_cuda(cudaMalloc(&bufs->model, GT_MAC_MODEL_FLOATS * sizeof(float)), "cudaMalloc");
                check_cuda(cudaMemcpy(bufs->model, o.mac_model, GT_MAC_MODEL_FLOATS * sizeof(float),
                                      cudaMemcpyHostToDevice), "model h2d");
            }
            rq.mac_model = bufs->model;
        } else {
            // the model is a small host array: stage it with the call
            rq.mac_model = stage_in(ctx, kSlotIn2, o.mac_model, (int64_t)GT_MAC_MODEL_FLOATS, GT_MEM_HOST);
        }
        rq.mac_kappa = o.mac_kappa;
        rq.mac_band_lo = o.mac_band[0];
        rq.mac_band_hi = o.mac_band[1];
    }
    rq.count = o.count != 0;
    rq.block_warps = o.block_warps;
    rq.list_capacity = o.list_capacity;
    rq.stack_capacity = o.stack_capacity;
    rq.pair_windows = o.no_window_pairs == 0;
    rq.bufs = bufs;
    rq.capture = capture;
    rq.sink_radius = o.sink_direct_radius;
    if ((ax == nullptr) != (ay == nullptr) || (ax == nullptr) != (az == nullptr))
        throw Fail{GT_ERR_INVALID, "ax, ay, az must all be given or all be null"};
    if (!ax && !phi && !tidal && !jerk) return;
    rq.ax = out_buf(ctx, kSlotOut0, ax, nout, mem);
    rq.ay = out_buf(ctx, kSlotOut1, ay, nout, mem);
    rq.az = out_buf(ctx, kSlotOut2, az, nout, mem);
    rq.phi = out_buf(ctx, kSlotOut3, phi, nout, mem);
    rq.tidal = out_buf(ctx, kSlotOut4, tidal, nout * 6, mem);
    rq.jerk = out_buf(ctx, kSlotOut5, jerk, nout * 3, mem);
    if (rq.out_original && nout > nt) {
        // massless particles are not walked; their outputs are defined as 0
        for (double* p : {rq.ax, rq.ay, rq.az, rq.phi})
            if (p) check_cuda(cudaMemsetAsync(p, 0, (size_t)nout * 8, ctx->stream), "memset");
        if (rq.tidal) check_cuda(cudaMemsetAsync(rq.tidal, 0, (size_t)nout * 48, ctx->stream), "memset");
        if (rq.jerk) check_cuda(cudaMemsetAsync(rq.jerk, 0, (size_t)nout * 24, ctx->stream), "memset");
    }
    // host outputs in target order: the walk copies each chunk back while the next one runs
    if (mem == GT_MEM_HOST && !rq.out_original && !capture) {
        rq.host.ax = ax; rq.host.ay = ay; rq.host.az = az;
        rq.host.phi = phi; rq.host.tidal = tidal; rq.host.jerk = jerk;
    }
    const bool copied = run_walk(ctx, tree, rq);
    if (capture) return;
    const bool sync_call = mem == GT_MEM_HOST || !o.async;
    uint32_t* bad_host = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->pinned) + kPinnedTargetCheck);
    if (!all && nt > 0 && sync_call) {
        *bad_host = 0;
        check_cuda(cudaMemcpyAsync(bad_host, (uint32_t*)scratch(ctx, kSlotGroupCount, 64) + 2, 4,
                                   cudaMemcpyDeviceToHost, ctx->stream), "target check d2h");
    }
    if (!copied) {
        copy_out(ctx, ax, rq.ax, nout, mem);
        copy_out(ctx, ay, rq.ay, nout, mem);
        copy_out(ctx, az, rq.az, nout, mem);
        copy_out(ctx, phi, rq.phi, nout, mem);
        copy_out(ctx, tidal, rq.tidal, nout * 6, mem);
        copy_out(ctx, jerk, rq.jerk, nout * 3, mem);
    }
    const bool sync = sync_call;
    finish(ctx, sync);
    if (sync) record_walk_time(ctx);
    if (!all && nt > 0 && sync && *bad_host) throw Fail{GT_ERR_INVALID, "target index out of range"};
}

}  // namespace

extern "C" {

int gt_version(void) { return GT_VERSION; }

const char* gt_status_string(int s) {
    switch (s) {
        case GT_OK: return "GT_OK";
        case GT_ERR_INVALID: return "GT_ERR_INVALID";
        case GT_ERR_CUDA: return "GT_ERR_CUDA";
        case GT_ERR_NOMEM: return "GT_ERR_NOMEM";
        case GT_ERR_UNSUPPORTED: return "GT_ERR_UNSUPPORTED";
        case GT_ERR_OVERFLOW: return "GT_ERR_OVERFLOW";
        case GT_ERR_TIMEOUT: return "GT_ERR_TIMEOUT";
        case GT_ERR_NONFINITE: return "GT_ERR_NONFINITE";
        case GT_ERR_DEVICE: return "GT_ERR_DEVICE";
        default: return "GT_ERR_UNKNOWN";
    }
}

void gt_build_options_default(gt_build_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->key_mode = GT_KEY_PEANO;
    o->leaf_max = 16;
    o->max_level = 20;
    o->randomize_seed = -1;
    o->nodelta = 0;
    o->validate = 1;
}

void gt_walk_options_default(gt_walk_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->group_mode = GT_GROUP_LEAF;
    o->group_max = 32;
    o->mac = GT_MAC_PLAIN;
    o->out_order = GT_OUT_TARGETS;
}

int gt_context_create(int device, gt_context** out) {
    if (!out) return GT_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        return GT_ERR_DEVICE;
    }
    if (device < 0 || device >= ndev) return GT_ERR_DEVICE;
    gt_context* ctx = new gt_context();
    ctx->device = device;
    const int st = guarded(ctx, [&] {
        DeviceGuard dg(device);
        cudaDeviceProp prop;
        check_cuda(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
        ctx->num_sms = prop.multiProcessorCount;
        check_cuda(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        // keep freed tree memory in this process's default pool of the device, so a tree rebuilt
        // every step reuses it instead of returning it to the driver at each synchronisation
        cudaMemPool_t pool;
        check_cuda(cudaDeviceGetDefaultMemPool(&pool, device), "cudaDeviceGetDefaultMemPool");
        uint64_t keep = UINT64_MAX;
        check_cuda(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep),
                   "cudaMemPoolSetAttribute");
        ctx->own_stream = true;
        check_cuda(cudaMallocHost(&ctx->pinned, 4096), "cudaMallocHost");
        check_cuda(cudaEventCreate(&ctx->ev0), "cudaEventCreate");
        check_cuda(cudaEventCreate(&ctx->ev1), "cudaEventCreate");
        ctx->scratch.resize(kSlotCount);
    });
    if (st != GT_OK) {
        gt_context_destroy(ctx);
        return st;
    }
    *out = ctx;
    return GT_OK;
}

int gt_context_destroy(gt_context* ctx) {
    if (!ctx) return GT_ERR_INVALID;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->scratch)
        if (b.ptr) cudaFree(b.ptr);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    for (cudaEvent_t e : ctx->chunk_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->up_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->down_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->stage) cudaFreeHost(ctx->stage);
    if (ctx->copy_done) cudaEventDestroy(ctx->copy_done);
    if (ctx->main_ev) cudaEventDestroy(ctx->main_ev);
    if (ctx->walk2) {
        cudaStreamSynchronize(ctx->walk2);
        cudaStreamDestroy(ctx->walk2);
    }
    if (ctx->walk2_start) cudaEventDestroy(ctx->walk2_start);
    if (ctx->tally_dev) cudaFree(ctx->tally_dev);
    if (ctx->walk2_done) cudaEventDestroy(ctx->walk2_done);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    delete ctx;
    return GT_OK;
}

const char* gt_last_error(const gt_context* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int gt_context_get_stream(gt_context* ctx, void** stream) {
    if (!ctx || !stream) return GT_ERR_INVALID;
    *stream = (void*)ctx->stream;
    return GT_OK;
}

int gt_context_set_stream(gt_context* ctx, void* stream) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        DeviceGuard dg(ctx->device);
        check_cuda(cudaStreamSynchronize(ctx->stream), "sync");
        if (ctx->own_stream) cudaStreamDestroy(ctx->stream);
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    });
}

int gt_synchronize(gt_context* ctx) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        DeviceGuard dg(ctx->device);
        check_cuda(cudaStreamSynchronize(ctx->stream), "cudaStreamSynchronize");
    });
}

int gt_launch_count(const gt_context* ctx, uint64_t* count) {
    if (!ctx || !count) return GT_ERR_INVALID;
    *count = ctx->launches;
    return GT_OK;
}

namespace {
int build_common(gt_context* ctx, int64_t n, int32_t n_systems, const int64_t* offsets, const double* x,
                 const double* y, const double* z, const double* m, const double* soft, int mem,
                 const gt_build_options* opt, gt_tree** out) {
    if (!ctx || !out) return GT_ERR_INVALID;
    *out = nullptr;
    gt_tree* t = new gt_tree();
    const int st = guarded(ctx, [&] {
        check_mem(mem);
        if (n < 0) throw Fail{GT_ERR_INVALID, "n < 0"};
        if (n > 0 && (!x || !y || !z || !m)) throw Fail{GT_ERR_INVALID, "null particle array"};
        if (n >= (int64_t)INT32_MAX) throw Fail{GT_ERR_INVALID, "n must be below 2^31"};
        if (n_systems < 1 || n_systems > (1 << 24)) throw Fail{GT_ERR_INVALID, "n_systems must be in [1, 2^24]"};
        if (n_systems > 1) {
            if (!offsets) throw Fail{GT_ERR_INVALID, "null system offsets"};
            if (offsets[0] != 0 || offsets[n_systems] != n)
                throw Fail{GT_ERR_INVALID, "system offsets must start at 0 and end at n"};
            for (int32_t s = 0; s < n_systems; ++s)
                if (offsets[s + 1] < offsets[s]) throw Fail{GT_ERR_INVALID, "system offsets must not decrease"};
        }
        gt_build_options o;
        gt_build_options_default(&o);
        if (opt) o = *opt;
        if (o.key_mode != GT_KEY_PEANO && o.key_mode != GT_KEY_MORTON) throw Fail{GT_ERR_INVALID, "unknown key_mode"};
        if (o.leaf_max < 1) throw Fail{GT_ERR_INVALID, "leaf_max < 1"};
        if (o.max_level < 1 || o.max_level > 20) throw Fail{GT_ERR_INVALID, "max_level must be in [1, 20]"};
        DeviceGuard dg(ctx->device);
        t->device = ctx->device;
        t->n = n;
        t->opt = o;
        const double* dx = stage_in(ctx, kSlotIn0, x, n, mem);
        const double* dy = stage_in(ctx, kSlotIn1, y, n, mem);
        const double* dz = stage_in(ctx, kSlotIn2, z, n, mem);
        const double* dm = stage_in(ctx, kSlotIn3, m, n, mem);
        const double* ds = nullptr;
        cudaEvent_t soft_ready = nullptr;
        if (mem == GT_MEM_HOST && soft && n > 0) {
            // the softenings are first read in the gather stage: upload them on the copy stream
            // once x, y, z, m are across, while the bounding box, keys and sort run
            ensure_copy_stream(ctx);
            double* d = (double*)scratch(ctx, kSlotIn4, (size_t)n * sizeof(double));
            check_cuda(cudaEventRecord(ctx->main_ev, ctx->stream), "event");
            check_cuda(cudaStreamWaitEvent(ctx->copy_stream, ctx->main_ev, 0), "wait");
            check_cuda(cudaMemcpyAsync(d, soft, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->copy_stream),
                       "H2D");
            check_cuda(cudaEventRecord(ctx->copy_done, ctx->copy_stream), "event");
            soft_ready = ctx->copy_done;
            ds = d;
        } else {
            ds = stage_in(ctx, kSlotIn4, soft, n, mem);
        }
        build_tree(ctx, t, dx, dy, dz, dm, ds, n_systems, offsets, soft_ready);
        finish(ctx, true);
    });
    if (st != GT_OK) {
        cudaStreamSynchronize(ctx->stream);  // queued build work may still use the arrays
        if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);  // and the softenings' upload
        cudaGetLastError();
        free_tree_arrays(t);
        delete t;
        return st;
    }
    *out = t;
    return GT_OK;
}
}  // namespace

int gt_build(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
             const double* m, const double* soft, int mem, const gt_build_options* opt,
             gt_tree** out) {
    return build_common(ctx, n, 1, nullptr, x, y, z, m, soft, mem, opt, out);
}

int gt_build_systems(gt_context* ctx, int64_t n, int32_t n_systems, const int64_t* offsets,
                     const double* x, const double* y, const double* z, const double* m,
                     const double* soft, int mem, const gt_build_options* opt, gt_tree** out) {
    return build_common(ctx, n, n_systems, offsets, x, y, z, m, soft, mem, opt, out);
}

int gt_tree_systems(const gt_tree* t, int64_t* live_offsets, double* roots) {
    if (!t) return GT_ERR_INVALID;
    for (int s = 0; s < t->n_systems; ++s) {
        if (live_offsets) live_offsets[s] = t->sys_off[s];
        if (roots) {
            const gt::RootGeom& g = t->sys_geom[s];
            roots[4 * s] = g.cx; roots[4 * s + 1] = g.cy; roots[4 * s + 2] = g.cz; roots[4 * s + 3] = g.side;
        }
    }
    if (live_offsets) live_offsets[t->n_systems] = t->sys_off[t->n_systems];
    return GT_OK;
}

int gt_tree_free(gt_tree* t) {
    if (!t) return GT_ERR_INVALID;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(t->device);
    cudaDeviceSynchronize();
    free_tree_arrays(t);
    cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    delete t;
    return GT_OK;
}

int gt_tree_info_get(const gt_tree* t, gt_tree_info* info) {
    if (!t || !info) return GT_ERR_INVALID;
    std::memset(info, 0, sizeof(*info));
    info->n = t->n;
    info->n_live = t->n_live;
    info->n_nodes = t->n_nodes;
    info->n_levels = t->n_levels;
    info->root = 0;
    info->center[0] = t->geom.cx;
    info->center[1] = t->geom.cy;
    info->center[2] = t->geom.cz;
    info->side = t->geom.side;
    for (int k = 0; k < 7; ++k) info->build_ms[k] = t->build_ms[k];
    info->n_systems = t->n_systems;
    return GT_OK;
}

int gt_tree_download(gt_context* ctx, const gt_tree* t, uint32_t* orderbuf, uint32_t* rank,
                     int32_t* leaf_of, const gt_node_arrays* nd) {
    if (!ctx || !t) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        DeviceGuard dg(ctx->device);
        cudaStream_t st = ctx->stream;
        const int64_t n = t->n, nl = t->n_live, nn = t->n_nodes;
        if (orderbuf && nl > 0)
            check_cuda(cudaMemcpyAsync(orderbuf, t->order, (size_t)nl * 4, cudaMemcpyDeviceToHost, st), "D2H");
        if (rank && n > 0)
            check_cuda(cudaMemcpyAsync(rank, t->rank, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "D2H");
        if (leaf_of && n > 0)
            check_cuda(cudaMemcpyAsync(leaf_of, t->leaf_of, (size_t)n * 4, cudaMemcpyDeviceToHost, st), "D2H");
        std::vector<GNode> hn;
        std::vector<double> hgc;
        if (nd) {
            hn.resize((size_t)nn);
            check_cuda(cudaMemcpyAsync(hn.data(), t->nodes, (size_t)nn * sizeof(GNode), cudaMemcpyDeviceToHost, st), "D2H");
            auto cp = [&](void* dst, const void* src, size_t bytes) {
                if (dst) check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st), "D2H");
            };
            cp(nd->size, t->size, (size_t)nn * 8);
            cp(nd->delta, t->delta, (size_t)nn * 8);
            cp(nd->soft, t->nsoft, (size_t)nn * 8);
            cp(nd->next, t->next, (size_t)nn * 4);
            cp(nd->parent, t->parent, (size_t)nn * 4);
            cp(nd->level, t->level, (size_t)nn * 4);
            if (nd->gcx || nd->gcy || nd->gcz) {
                hgc.resize((size_t)nn * 3);
                check_cuda(cudaMemcpyAsync(hgc.data(), t->gc, (size_t)nn * 24, cudaMemcpyDeviceToHost, st), "D2H");
            }
        }
        check_cuda(cudaStreamSynchronize(st), "sync");
        if (rank)  // the reference marks massless particles with UINT32_MAX
            for (int64_t i = 0; i < n; ++i)
                if ((int64_t)rank[i] >= nl) rank[i] = UINT32_MAX;
        if (nd) {
            for (int64_t i = 0; i < nn; ++i) {
                const GNode& g = hn[(size_t)i];
                if (nd->cx) nd->cx[i] = g.cx;
                if (nd->cy) nd->cy[i] = g.cy;
                if (nd->cz) nd->cz[i] = g.cz;
                if (nd->mass) nd->mass[i] = g.mass;
                if (nd->first) nd->first[i] = g.first;
                if (nd->plo) nd->plo[i] = g.plo;
                if (nd->phi) nd->phi[i] = g.phi;
                if (nd->w_s) nd->w_s[i] = g.s;
                if (nd->w_len) nd->w_len[i] = g.len;
                if (nd->w_soft) nd->w_soft[i] = g.soft;
                if (nd->gcx) nd->gcx[i] = hgc[3 * i];
                if (nd->gcy) nd->gcy[i] = hgc[3 * i + 1];
                if (nd->gcz) nd->gcz[i] = hgc[3 * i + 2];
            }
        }
    });
}

int gt_tree_keys(gt_context* ctx, const gt_tree* t, uint64_t* keys) {
    if (!ctx || !t || !keys) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        DeviceGuard dg(ctx->device);
        if (t->n_live > 0)
            check_cuda(cudaMemcpyAsync(keys, t->skey, (size_t)t->n_live * 8, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        finish(ctx, true);
    });
}

int gt_accel_grouped(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
                     const double* aold, double theta, double G, int batch, const gt_walk_options* opt,
                     int mem, double* ax, double* ay, double* az, double* phi) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        gt_walk_options o;
        gt_walk_options_default(&o);
        if (opt) o = *opt;
        int mode = o.group_mode, param = 0;
        if (mode == GT_GROUP_LEAF && batch > 0) mode = GT_GROUP_BATCH;
        if (mode == GT_GROUP_BATCH) param = batch > 0 ? batch : 8;
        if (mode == GT_GROUP_NODE) param = o.group_max;
        if (mode < GT_GROUP_LEAF || mode > GT_GROUP_SINGLE) throw Fail{GT_ERR_INVALID, "unknown group_mode"};
        walk_common(ctx, tree, n_targets, targets, aold, theta, G, mode, param, true, &o, mem, ax, ay, az, phi);
    });
}

void gt_tune_options_default(gt_tune_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->reps = 3;
    o->p99_max = 5e-3;
}

int gt_autotune(gt_context* ctx, const gt_tree* tree, const double* aold, int mem, double theta, double G,
                const gt_tune_options* opt, gt_walk_options* best, int* best_batch, gt_tune_entry* entries,
                int max_entries, int* n_entries) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree || !best) throw Fail{GT_ERR_INVALID, "null tree or output"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
        gt_tune_options o;
        gt_tune_options_default(&o);
        if (opt) o = *opt;
        if (o.n_sample < 0 || (o.n_sample > 0 && (!o.sample || !o.ref_ax || !o.ref_ay || !o.ref_az)))
            throw Fail{GT_ERR_INVALID, "bad sample"};
        for (int64_t i = 0; i < o.n_sample; ++i)
            if ((int64_t)o.sample[i] >= tree->n) throw Fail{GT_ERR_INVALID, "sample index out of range"};
        if (o.mac_model && (o.n_kappa <= 0 || !o.kappa)) throw Fail{GT_ERR_INVALID, "a model needs kappa values"};
        DeviceGuard dg(ctx->device);
        TuneRequest tr;
        tr.reps = o.reps;
        tr.p99_max = o.p99_max;
        tr.n_sample = o.n_sample;
        tr.sample = o.sample;
        tr.ref_ax = o.ref_ax; tr.ref_ay = o.ref_ay; tr.ref_az = o.ref_az;
        if (o.mac_model) {
            tr.mac_model = stage_in(ctx, kSlotIn2, o.mac_model, (int64_t)GT_MAC_MODEL_FLOATS, GT_MEM_HOST);
            tr.kappa.assign(o.kappa, o.kappa + o.n_kappa);
            tr.mac_band[0] = o.mac_band[0];
            tr.mac_band[1] = o.mac_band[1];
            tr.mac_mode = o.mac_mode == GT_MAC_NODE ? GT_MAC_NODE : GT_MAC_LEARNED;
            if (o.mac_mode != 0 && o.mac_mode != GT_MAC_LEARNED && o.mac_mode != GT_MAC_NODE)
                throw Fail{GT_ERR_INVALID, "unknown mac_mode"};
        }
        const double* da = stage_in(ctx, kSlotIn1, aold, tree->n_live, mem);
        std::vector<gt_tune_entry> all;
        gt_tune_entry b;
        run_autotune(ctx, tree, da, theta, G, tr, all, b);
        gt_walk_options w;
        gt_walk_options_default(&w);
        w.group_mode = b.group_mode;
        if (b.group_mode == GT_GROUP_NODE) w.group_max = b.group_size;
        w.block_warps = b.block_warps;
        w.list_capacity = b.list_capacity;
        w.mac = b.mac;
        if (b.mac != GT_MAC_PLAIN) {
            w.mac_model = o.mac_model;
            w.mac_kappa = b.mac_kappa;
            w.mac_band[0] = o.mac_band[0];
            w.mac_band[1] = o.mac_band[1];
        }
        *best = w;
        if (best_batch) *best_batch = b.group_mode == GT_GROUP_BATCH ? b.group_size : 0;
        const int k = (int)std::min<size_t>(all.size(), (size_t)std::max(0, max_entries));
        if (entries)
            for (int i = 0; i < k; ++i) entries[i] = all[i];
        if (n_entries) *n_entries = entries ? k : (int)all.size();
    });
}

int gt_accel_grouped_ext(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
                         const double* aold, double theta, double G, int batch, const gt_walk_options* opt,
                         int mem, double* ax, double* ay, double* az, double* phi, double* tidal,
                         double* jerk) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        gt_walk_options o;
        gt_walk_options_default(&o);
        if (opt) o = *opt;
        int mode = o.group_mode, param = 0;
        if (mode == GT_GROUP_LEAF && batch > 0) mode = GT_GROUP_BATCH;
        if (mode == GT_GROUP_BATCH) param = batch > 0 ? batch : 8;
        if (mode == GT_GROUP_NODE) param = o.group_max;
        if (mode < GT_GROUP_LEAF || mode > GT_GROUP_NODE) throw Fail{GT_ERR_INVALID, "unknown group_mode"};
        walk_common(ctx, tree, n_targets, targets, aold, theta, G, mode, param, true, &o, mem, ax, ay, az, phi,
                    nullptr, false, tidal, jerk);
    });
}

int gt_tree_velocities(gt_context* ctx, gt_tree* tree, const double* vx, const double* vy, const double* vz,
                       int particles_only, int mem) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree || (tree->n > 0 && (!vx || !vy || !vz))) throw Fail{GT_ERR_INVALID, "null tree or velocity"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
        DeviceGuard dg(ctx->device);
        const double* dx = stage_in(ctx, kSlotIn0, vx, tree->n, mem);
        const double* dy = stage_in(ctx, kSlotIn1, vy, tree->n, mem);
        const double* dz = stage_in(ctx, kSlotIn2, vz, tree->n, mem);
        if (particles_only && !tree->svel) throw Fail{GT_ERR_INVALID, "no node velocities to keep yet"};
        tree_velocities(ctx, tree, dx, dy, dz, particles_only != 0);
        finish(ctx, true);
    });
}

int gt_tree_gas(gt_context* ctx, gt_tree* tree, const uint8_t* type, const double* zeta, int mem) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree) throw Fail{GT_ERR_INVALID, "null tree"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
        if (mem == GT_MEM_HOST && zeta && tree->opt.validate)
            for (int64_t i = 0; i < tree->n; ++i)
                if (!std::isfinite(zeta[i])) throw Fail{GT_ERR_NONFINITE, "non-finite zeta"};
        DeviceGuard dg(ctx->device);
        const uint8_t* dt = stage_in(ctx, kSlotIn0, type, tree->n, mem);
        const double* dz = stage_in(ctx, kSlotIn1, zeta, tree->n, mem);
        tree_gas(ctx, tree, dt, dz);
        finish(ctx, true);
    });
}

int gt_tree_events(gt_context* ctx, gt_tree* tree, int kind, int64_t n, const int32_t* leaf, const double* a,
                   const double* x, const double* v, const float* f, double tau, double box, int mem) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree || n < 0) throw Fail{GT_ERR_INVALID, "null tree or negative count"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
        if (kind < GT_EVENT_KICK || kind > GT_EVENT_HMAX) throw Fail{GT_ERR_INVALID, "unknown event kind"};
        if (n == 0) return;
        const bool need_a = kind != GT_EVENT_VMAX, need_x = kind == GT_EVENT_SHIFT || kind == GT_EVENT_MASS;
        if (!leaf || (need_a && !a) || (need_x && !x) || (kind == GT_EVENT_MASS && !v) ||
            (kind == GT_EVENT_VMAX && !f))
            throw Fail{GT_ERR_INVALID, "null event array"};
        if (mem == GT_MEM_HOST)
            for (int64_t e = 0; e < n; ++e)
                if (leaf[e] >= (int64_t)tree->n_nodes) throw Fail{GT_ERR_INVALID, "leaf node out of range"};
        DeviceGuard dg(ctx->device);
        const int* dl = stage_in(ctx, kSlotIn0, leaf, n, mem);
        const double* da = need_a ? stage_in(ctx, kSlotIn1, a, kind == GT_EVENT_KICK ? 3 * n : n, mem) : nullptr;
        const double* dx = need_x ? stage_in(ctx, kSlotIn2, x, 3 * n, mem) : nullptr;
        const double* dv = kind == GT_EVENT_MASS ? stage_in(ctx, kSlotIn3, v, 3 * n, mem) : nullptr;
        const float* df = kind == GT_EVENT_VMAX ? stage_in(ctx, kSlotIn4, f, n, mem) : nullptr;
        if (kind == GT_EVENT_HMAX) raise_hmax(ctx, tree, n, dl, da);
        else reuse_events(ctx, tree, kind, n, dl, da, dx, dv, df, tau, box);
        finish(ctx, mem == GT_MEM_HOST);
    });
}

void gt_ngb_options_default(gt_ngb_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->mode = GT_NGB_GATHER;
}

void gt_density_options_default(gt_density_options* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->des_ngb = 32.0;
    o->ngb_tol = 0.05;
    o->n_dims = 3;
    o->face_correction = 1;
}

int gt_tree_hmax(gt_context* ctx, gt_tree* tree, const double* h, int64_t n_gas, int mem) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree || n_gas < 0 || (n_gas > 0 && !h)) throw Fail{GT_ERR_INVALID, "null tree or h, or n_gas < 0"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
        DeviceGuard dg(ctx->device);
        const int64_t n = std::min<int64_t>(n_gas, tree->n);
        tree_hmax(ctx, tree, stage_in(ctx, kSlotIn0, h, n, mem), n);
        finish(ctx, true);
    });
}

int gt_ngb_search(gt_context* ctx, const gt_tree* tc, int64_t n, const double* cx, const double* cy,
                  const double* cz, const double* radius, const gt_ngb_options* opt, int mem, int64_t* start,
                  uint32_t* found, int64_t capacity, int64_t* total) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        gt_tree* tree = const_cast<gt_tree*>(tc);  // search nodes are made on first use
        if (!tree || n < 0 || !start) throw Fail{GT_ERR_INVALID, "null tree or start, or n < 0"};
        if (n > 0 && (!cx || !cy || !cz || !radius)) throw Fail{GT_ERR_INVALID, "null centre or radius"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
        gt_ngb_options o;
        gt_ngb_options_default(&o);
        if (opt) o = *opt;
        if (o.mode < GT_NGB_GATHER || o.mode > GT_NGB_PAIRS) throw Fail{GT_ERR_INVALID, "unknown search mode"};
        if (o.mode != GT_NGB_GATHER && o.n_gas > 0 && !o.h) throw Fail{GT_ERR_INVALID, "the reverse search needs h"};
        if (!(o.box >= 0.0) || !(o.elapsed >= 0.0)) throw Fail{GT_ERR_INVALID, "box and elapsed must be >= 0"};
        if (capacity < 0) throw Fail{GT_ERR_INVALID, "capacity < 0"};
        DeviceGuard dg(ctx->device);
        if (total) *total = 0;
        if (n == 0) {
            start[0] = 0;  // host or device: one int64
            if (mem == GT_MEM_DEVICE) check_cuda(cudaMemsetAsync(start, 0, 8, ctx->stream), "memset");
            finish(ctx, true);
            return;
        }
        const double* dx = stage_in(ctx, kSlotIn0, cx, n, mem);
        const double* dy = stage_in(ctx, kSlotIn1, cy, n, mem);
        const double* dz = stage_in(ctx, kSlotIn2, cz, n, mem);
        const double* dr = stage_in(ctx, kSlotIn3, radius, n, mem);
        const int64_t ng = o.mode == GT_NGB_GATHER ? 0 : std::min<int64_t>(o.n_gas, tree->n);
        const double* dh = stage_in(ctx, kSlotIn4, o.h, ng, mem);
        const int* dsys = (const int*)stage_in(ctx, kSlotIn5, o.systems, n, mem);
        int64_t* ds = out_buf(ctx, kSlotOut0, start, n + 1, mem);
        // the host path makes the lists in a workspace buffer once the counting pass has sized
        // them.  SHMEM_NGB_COUNT: a call counts its searches once, when it delivers the lists; a
        // count-only call or one that overflows counts nothing, so counting then filling counts
        // each search once
        uint32_t* df = mem == GT_MEM_DEVICE ? found : nullptr;
        int64_t tl[5] = {0, 0, 0, 0, 0};
        const bool counted = ctx->ngb_count && found;
        uint32_t* hf = nullptr;  // host path: the lists, made on the device in one call
        const int64_t tot = run_ngb(ctx, tree, n, dx, dy, dz, dr, dsys, o.mode, dh, ng, o.box, o.elapsed, ds, df,
                                    found ? capacity : 0, counted ? tl : nullptr,
                                    mem == GT_MEM_HOST && found ? &hf : nullptr);
        if (total) *total = tot;
        copy_out(ctx, start, ds, n + 1, mem);
        if (hf) copy_out(ctx, found, hf, tot, mem);
        finish(ctx, true);
        if (found && tot > capacity) throw Fail{GT_ERR_OVERFLOW, "the neighbour lists need more room than capacity"};
        if (counted)
            for (int k = 0; k < 5; ++k) ctx->ngb_totals[k] += tl[k];
    });
}

int gt_density(gt_context* ctx, const gt_tree* tc, int64_t nt, const uint32_t* targets,
               const gt_density_options* opt, int mem, double* h, double* rho, int32_t* nngb, int32_t* iters) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        gt_tree* tree = const_cast<gt_tree*>(tc);
        if (!tree || nt < 0 || (nt > 0 && !targets)) throw Fail{GT_ERR_INVALID, "null tree or targets, or nt < 0"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "tree and context are on different devices"};
        gt_density_options o;
        gt_density_options_default(&o);
        if (opt) o = *opt;
        if (o.n_dims < 1 || o.n_dims > 3) throw Fail{GT_ERR_INVALID, "n_dims must be 1, 2 or 3"};
        if (!(o.des_ngb > 0.0) || !(o.ngb_tol > 0.0)) throw Fail{GT_ERR_INVALID, "des_ngb and ngb_tol must be > 0"};
        if (!(o.box >= 0.0) || !(o.elapsed >= 0.0)) throw Fail{GT_ERR_INVALID, "box and elapsed must be >= 0"};
        if (mem == GT_MEM_HOST)
            for (int64_t k = 0; k < nt; ++k)
                if ((int64_t)targets[k] >= tree->n) throw Fail{GT_ERR_INVALID, "target index out of range"};
        DeviceGuard dg(ctx->device);
        if (nt == 0) return;
        const uint32_t* dt = stage_in(ctx, kSlotIn0, targets, nt, mem);
        const double* dhs = stage_in(ctx, kSlotIn1, o.h_start, nt, mem);
        const double* dcp = stage_in(ctx, kSlotIn2, o.cond_prev, tree->n, mem);
        double* dh = (double*)(mem == GT_MEM_DEVICE && h ? (void*)h : scratch(ctx, kSlotOut0, (size_t)nt * 8));
        double* dr = (double*)(mem == GT_MEM_DEVICE && rho ? (void*)rho : scratch(ctx, kSlotOut1, (size_t)nt * 8));
        int* dn = (int*)(mem == GT_MEM_DEVICE && nngb ? (void*)nngb : scratch(ctx, kSlotOut2, (size_t)nt * 4));
        int* di = (int*)(mem == GT_MEM_DEVICE && iters ? (void*)iters : scratch(ctx, kSlotOut3, (size_t)nt * 4));
        int64_t tl[GT_NGB_COUNTERS] = {};
        run_density(ctx, tree, nt, dt, o.des_ngb, o.ngb_tol, dhs, o.box, o.n_dims, dcp, o.face_correction != 0,
                    o.elapsed, dh, dr, dn, di, ctx->ngb_count ? tl : nullptr);
        copy_out(ctx, h, dh, nt, mem);
        copy_out(ctx, rho, dr, nt, mem);
        copy_out(ctx, nngb, (int32_t*)dn, nt, mem);
        copy_out(ctx, iters, (int32_t*)di, nt, mem);
        finish(ctx, true);
        if (ctx->ngb_count)
            for (int k = 0; k < GT_NGB_COUNTERS; ++k) ctx->ngb_totals[k] += tl[k];
    });
}

int gt_ngb_count(gt_context* ctx, int enable) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        ctx->ngb_count = enable != 0;
    });
}

int gt_ngb_counters_get(gt_context* ctx, int64_t* counts, int reset) {
    if (!ctx || !counts) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        for (int k = 0; k < GT_NGB_COUNTERS; ++k) {
            counts[k] = ctx->ngb_totals[k];
            if (reset) ctx->ngb_totals[k] = 0;
        }
    });
}

int gt_tree_refresh(gt_context* ctx, gt_tree* tree, double tau) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        if (!tree) throw Fail{GT_ERR_INVALID, "null tree"};
        DeviceGuard dg(ctx->device);
        reuse_refresh(ctx, tree, tau);
        finish(ctx, true);
    });
}

int gt_tree_node_state(gt_context* ctx, gt_tree* tree, double tau, double* com, double* vel, double* mass,
                       float* vmax, float* xpad) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        if (!tree) throw Fail{GT_ERR_INVALID, "null tree"};
        DeviceGuard dg(ctx->device);
        const int64_t nn = tree->n_nodes;
        double* dcom = (double*)scratch(ctx, kSlotOut0, (size_t)std::max<int64_t>(nn, 1) * 24);
        double* dvel = (double*)scratch(ctx, kSlotOut1, (size_t)std::max<int64_t>(nn, 1) * 24);
        double* dmass = (double*)scratch(ctx, kSlotOut2, (size_t)std::max<int64_t>(nn, 1) * 8);
        reuse_node_state(ctx, tree, tau, dcom, dvel, dmass);
        copy_out(ctx, com, (const double*)dcom, 3 * nn, GT_MEM_HOST);
        copy_out(ctx, vel, (const double*)dvel, 3 * nn, GT_MEM_HOST);
        copy_out(ctx, mass, (const double*)dmass, nn, GT_MEM_HOST);
        copy_out(ctx, vmax, (const float*)tree->vmax, nn, GT_MEM_HOST);
        copy_out(ctx, xpad, (const float*)tree->xpad, nn, GT_MEM_HOST);
        finish(ctx, true);
    });
}

int gt_tree_particles(gt_context* ctx, gt_tree* tree, const double* x, const double* y, const double* z,
                      const double* m, const double* soft, int mem) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree) throw Fail{GT_ERR_INVALID, "null tree"};
        if ((x == nullptr) != (y == nullptr) || (x == nullptr) != (z == nullptr))
            throw Fail{GT_ERR_INVALID, "x, y, z must all be given or all be null"};
        DeviceGuard dg(ctx->device);
        const int64_t n = tree->n;
        tree_particles(ctx, tree, stage_in(ctx, kSlotIn0, x, n, mem), stage_in(ctx, kSlotIn1, y, n, mem),
                       stage_in(ctx, kSlotIn2, z, n, mem), stage_in(ctx, kSlotIn3, m, n, mem),
                       stage_in(ctx, kSlotIn4, soft, n, mem));
        finish(ctx, mem == GT_MEM_HOST);
    });
}

int gt_tree_velocity_moments(gt_context* ctx, const gt_tree* t, double* vcx, double* vcy, double* vcz,
                             float* vmax) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        if (!t) throw Fail{GT_ERR_INVALID, "null tree"};
        if (!t->vcom) throw Fail{GT_ERR_INVALID, "no velocities attached (gt_tree_velocities)"};
        DeviceGuard dg(ctx->device);
        const int64_t nn = t->n_nodes;
        std::vector<double> v((size_t)std::max<int64_t>(nn, 1) * 3);
        if (nn > 0) {
            check_cuda(cudaMemcpyAsync(v.data(), t->vcom, (size_t)nn * 24, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            if (vmax)
                check_cuda(cudaMemcpyAsync(vmax, t->vmax, (size_t)nn * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        }
        finish(ctx, true);
        for (int64_t i = 0; i < nn; ++i) {
            if (vcx) vcx[i] = v[3 * i];
            if (vcy) vcy[i] = v[3 * i + 1];
            if (vcz) vcz[i] = v[3 * i + 2];
        }
    });
}

int gt_plan_create(gt_context* ctx, const gt_tree* tree, const double* aold, double theta, double G, int batch,
                   const gt_walk_options* opt, double* ax, double* ay, double* az, double* phi, gt_plan** out) {
    if (!ctx || !out) return GT_ERR_INVALID;
    *out = nullptr;
    gt_plan* p = new gt_plan();
    p->ctx = ctx;
    p->tree = tree;
    bool capturing = false;
    // capture on a stream of our own: the context stream may be the legacy default stream, which
    // cannot be captured; replays go to the context stream
    cudaStream_t saved = ctx->stream, cs = nullptr;
    const int st = guarded(ctx, [&] {
        if (!tree) throw Fail{GT_ERR_INVALID, "null tree"};
        gt_walk_options o;
        gt_walk_options_default(&o);
        if (opt) o = *opt;
        if (o.count) throw Fail{GT_ERR_INVALID, "a plan does not collect counts"};
        if (o.stack_capacity) throw Fail{GT_ERR_INVALID, "a plan uses the default stack capacity"};
        o.async = 1;
        int mode = o.group_mode, param = 0;
        if (mode == GT_GROUP_LEAF && batch > 0) mode = GT_GROUP_BATCH;
        if (mode == GT_GROUP_BATCH) param = batch > 0 ? batch : 8;
        if (mode == GT_GROUP_NODE) param = o.group_max;
        if (mode < GT_GROUP_LEAF || mode > GT_GROUP_SINGLE) throw Fail{GT_ERR_INVALID, "unknown group_mode"};
        DeviceGuard dg(ctx->device);
        // one ordinary walk first: it builds the group list, sizes the plan's buffers and sets
        // the kernel attributes, so the capture below allocates nothing
        walk_common(ctx, tree, 0, nullptr, aold, theta, G, mode, param, true, &o, GT_MEM_DEVICE, ax, ay, az,
                    phi, &p->bufs, false);
        check_cuda(cudaStreamSynchronize(ctx->stream), "sync");
        const uint64_t before = ctx->launches;
        check_cuda(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "cudaStreamCreate");
        ctx->stream = cs;
        check_cuda(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        capturing = true;
        walk_common(ctx, tree, 0, nullptr, aold, theta, G, mode, param, true, &o, GT_MEM_DEVICE, ax, ay, az,
                    phi, &p->bufs, true);
        capturing = false;
        check_cuda(cudaStreamEndCapture(cs, &p->graph), "cudaStreamEndCapture");
        ctx->stream = saved;
        p->kernels = ctx->launches - before;
        ctx->launches = before;  // captured, not launched
        check_cuda(cudaGraphInstantiate(&p->exec, p->graph, 0), "cudaGraphInstantiate");
    });
    if (capturing) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
    }
    ctx->stream = saved;
    if (cs) cudaStreamDestroy(cs);
    if (st != GT_OK) {
        cudaGetLastError();
        gt_plan_destroy(p);
        return st;
    }
    *out = p;
    return GT_OK;
}

int gt_plan_launch(gt_plan* p) {
    if (!p || !p->exec) return GT_ERR_INVALID;
    return guarded(p->ctx, [&] {
        DeviceGuard dg(p->ctx->device);
        check_cuda(cudaGraphLaunch(p->exec, p->ctx->stream), "cudaGraphLaunch");
        p->ctx->launches += p->kernels;
    });
}

int gt_plan_destroy(gt_plan* p) {
    if (!p) return GT_ERR_INVALID;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(p->ctx->device);
    if (p->ctx->stream) cudaStreamSynchronize(p->ctx->stream);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    for (void* q : {(void*)p->bufs.stack, (void*)p->bufs.ctr, (void*)p->bufs.model})
        if (q) cudaFree(q);
    cudaGetLastError();
    if (prev >= 0) cudaSetDevice(prev);
    delete p;
    return GT_OK;
}

int gt_accel(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
             double theta, double G, const double* aold, int mem, double* ax, double* ay, double* az) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        walk_common(ctx, tree, n_targets, targets, aold, theta, G, GT_GROUP_SINGLE, 0, false, nullptr,
                    mem, ax, ay, az, nullptr);
    });
}

int gt_potential(gt_context* ctx, const gt_tree* tree, int64_t n_targets, const uint32_t* targets,
                 double theta, double G, const double* aold, int mem, double* phi) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        if (!phi) throw Fail{GT_ERR_INVALID, "phi is null"};
        walk_common(ctx, tree, n_targets, targets, aold, theta, G, GT_GROUP_SINGLE, 0, false, nullptr,
                    mem, nullptr, nullptr, nullptr, phi);
    });
}

int gt_walk_stats_get(const gt_context* ctx, gt_walk_stats* s) {
    if (!ctx || !s) return GT_ERR_INVALID;
    *s = ctx->stats;
    return GT_OK;
}

int gt_form_aold(gt_context* ctx, int64_t n, const double* ax, const double* ay, const double* az,
                 double alpha, double G, int mem, double* aold) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (n < 0 || (n > 0 && (!ax || !ay || !az || !aold))) throw Fail{GT_ERR_INVALID, "bad arguments"};
        if (!(G != 0.0)) throw Fail{GT_ERR_INVALID, "G must be non-zero"};
        DeviceGuard dg(ctx->device);
        const double* dx = stage_in(ctx, kSlotIn0, ax, n, mem);
        const double* dy = stage_in(ctx, kSlotIn1, ay, n, mem);
        const double* dz = stage_in(ctx, kSlotIn2, az, n, mem);
        double* o = out_buf(ctx, kSlotOut0, aold, n, mem);
        run_form_aold(ctx, n, dx, dy, dz, alpha, G, o);
        copy_out(ctx, aold, (const double*)o, n, mem);
        finish(ctx, true);
    });
}

int gt_direct_gas(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z, const double* m,
                  const double* soft, const uint8_t* type, const double* zeta, int64_t n_targets,
                  const uint32_t* targets, double G, int mem, double* ax, double* ay, double* az) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (n < 0 || n_targets < 0) throw Fail{GT_ERR_INVALID, "negative size"};
        if (n > 0 && (!x || !y || !z || !m)) throw Fail{GT_ERR_INVALID, "null source array"};
        if (n_targets > 0 && (!targets || !ax || !ay || !az)) throw Fail{GT_ERR_INVALID, "null targets or output"};
        if (mem == GT_MEM_HOST)
            for (int64_t k = 0; k < n_targets; ++k)
                if ((int64_t)targets[k] >= n) throw Fail{GT_ERR_INVALID, "target index out of range"};
        DeviceGuard dg(ctx->device);
        const double* dx = stage_in(ctx, kSlotIn0, x, n, mem);
        const double* dy = stage_in(ctx, kSlotIn1, y, n, mem);
        const double* dz = stage_in(ctx, kSlotIn2, z, n, mem);
        const double* dm = stage_in(ctx, kSlotIn3, m, n, mem);
        const double* ds = stage_in(ctx, kSlotIn4, soft, n, mem);
        const uint8_t* dty = stage_in(ctx, kSlotNodeTmp2, type, n, mem);
        const double* dze = stage_in(ctx, kSlotNodeTmp0, zeta, n, mem);
        const uint32_t* dt = stage_in(ctx, kSlotTargets, targets, n_targets, mem);
        double* oax = out_buf(ctx, kSlotOut0, ax, n_targets, mem);
        double* oay = out_buf(ctx, kSlotOut1, ay, n_targets, mem);
        double* oaz = out_buf(ctx, kSlotOut2, az, n_targets, mem);
        run_direct_gas(ctx, n, dx, dy, dz, dm, ds, dty, dze, n_targets, dt, G, oax, oay, oaz);
        copy_out(ctx, ax, (const double*)oax, n_targets, mem);
        copy_out(ctx, ay, (const double*)oay, n_targets, mem);
        copy_out(ctx, az, (const double*)oaz, n_targets, mem);
        finish(ctx, true);
    });
}

int gt_direct(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
              const double* m, const double* soft, int64_t n_targets, const uint32_t* targets,
              double G, int precision, int mem, double* ax, double* ay, double* az, double* phi) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (n < 0 || n_targets < 0) throw Fail{GT_ERR_INVALID, "negative size"};
        if (n > 0 && (!x || !y || !z || !m)) throw Fail{GT_ERR_INVALID, "null source array"};
        if (n_targets > 0 && !targets) throw Fail{GT_ERR_INVALID, "null targets"};
        if (precision != GT_DIRECT_FP64 && precision != GT_DIRECT_FP32) throw Fail{GT_ERR_INVALID, "unknown precision"};
        if (mem == GT_MEM_HOST)
            for (int64_t k = 0; k < n_targets; ++k)
                if ((int64_t)targets[k] >= n) throw Fail{GT_ERR_INVALID, "target index out of range"};
        DeviceGuard dg(ctx->device);
        const double* dx = stage_in(ctx, kSlotIn0, x, n, mem);
        const double* dy = stage_in(ctx, kSlotIn1, y, n, mem);
        const double* dz = stage_in(ctx, kSlotIn2, z, n, mem);
        const double* dm = stage_in(ctx, kSlotIn3, m, n, mem);
        const double* ds = stage_in(ctx, kSlotIn4, soft, n, mem);
        const uint32_t* dt = stage_in(ctx, kSlotTargets, targets, n_targets, mem);
        double* oax = out_buf(ctx, kSlotOut0, ax, n_targets, mem);
        double* oay = out_buf(ctx, kSlotOut1, ay, n_targets, mem);
        double* oaz = out_buf(ctx, kSlotOut2, az, n_targets, mem);
        double* oph = out_buf(ctx, kSlotOut3, phi, n_targets, mem);
        run_direct(ctx, n, dx, dy, dz, dm, ds, n_targets, dt, G, precision, oax, oay, oaz, oph);
        copy_out(ctx, ax, (const double*)oax, n_targets, mem);
        copy_out(ctx, ay, (const double*)oay, n_targets, mem);
        copy_out(ctx, az, (const double*)oaz, n_targets, mem);
        copy_out(ctx, phi, (const double*)oph, n_targets, mem);
        finish(ctx, true);
    });
}

int gt_peano_keys(gt_context* ctx, int64_t n, const double* x, const double* y, const double* z,
                  const double corner[3], double len, int bits, int mem, uint64_t* ph_hi,
                  uint64_t* ph_lo, uint64_t* mo_hi, uint64_t* mo_lo) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (n < 0 || !corner || !(len > 0)) throw Fail{GT_ERR_INVALID, "bad arguments"};
        if (bits < 1 || bits > 42) throw Fail{GT_ERR_INVALID, "bits must be in [1, 42]"};
        if (n > 0 && (!x || !y || !z)) throw Fail{GT_ERR_INVALID, "null coordinate array"};
        DeviceGuard dg(ctx->device);
        const double* dx = stage_in(ctx, kSlotIn0, x, n, mem);
        const double* dy = stage_in(ctx, kSlotIn1, y, n, mem);
        const double* dz = stage_in(ctx, kSlotIn2, z, n, mem);
        uint64_t* a = out_buf(ctx, kSlotOut0, ph_hi, n, mem);
        uint64_t* b = out_buf(ctx, kSlotOut1, ph_lo, n, mem);
        uint64_t* c = out_buf(ctx, kSlotOut2, mo_hi, n, mem);
        uint64_t* d = out_buf(ctx, kSlotOut3, mo_lo, n, mem);
        run_peano_keys(ctx, n, dx, dy, dz, corner, len, bits, a, b, c, d);
        copy_out(ctx, ph_hi, (const uint64_t*)a, n, mem);
        copy_out(ctx, ph_lo, (const uint64_t*)b, n, mem);
        copy_out(ctx, mo_hi, (const uint64_t*)c, n, mem);
        copy_out(ctx, mo_lo, (const uint64_t*)d, n, mem);
        finish(ctx, true);
    });
}

void gt_mac_train_options_default(gt_mac_train_options* o) {
    if (!o) return;
    o->epochs = 30;
    o->batch = 4096;
    o->lr = 2e-3;
    o->tau = 0.9;
    o->seed = 1;
    o->feature_mask = 0xFFu;
}

int gt_mac_sample(gt_context* ctx, const gt_tree* tree, const double* amag, double alpha, int window,
                  int64_t group_stride, double rho_lo, double rho_hi, int64_t capacity, int mem,
                  float* features, float* labels, float* rho, int64_t* n_samples) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree || !amag || !n_samples || capacity < 0) throw Fail{GT_ERR_INVALID, "bad arguments"};
        if (window < 1 || window > 32) throw Fail{GT_ERR_INVALID, "window must be in [1, 32]"};
        if (!(alpha > 0) || !(rho_hi >= rho_lo)) throw Fail{GT_ERR_INVALID, "bad alpha or rho window"};
        if (capacity > 0 && (!features || !labels || !rho)) throw Fail{GT_ERR_INVALID, "null output"};
        if (tree->n_systems > 1) throw Fail{GT_ERR_UNSUPPORTED, "gt_mac_sample takes a single-system tree"};
        DeviceGuard dg(ctx->device);
        const double* da = stage_in(ctx, kSlotIn0, amag, tree->n_live, mem);
        float* f = out_buf(ctx, kSlotOut0, features, capacity * GT_MAC_FEATURES, mem);
        float* l = out_buf(ctx, kSlotOut1, labels, capacity, mem);
        float* r = out_buf(ctx, kSlotOut2, rho, capacity, mem);
        run_mac_sample(ctx, tree, da, alpha, window, group_stride, rho_lo, rho_hi, capacity, f, l, r,
                       n_samples);
        const int64_t got = std::min(*n_samples, capacity);
        copy_out(ctx, features, (const float*)f, got * GT_MAC_FEATURES, mem);
        copy_out(ctx, labels, (const float*)l, got, mem);
        copy_out(ctx, rho, (const float*)r, got, mem);
        finish(ctx, true);
    });
}

int gt_tree_audit(gt_context* ctx, const gt_tree* tree, int64_t* n_bad, char* msg, size_t msglen) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        if (!tree || !n_bad) throw Fail{GT_ERR_INVALID, "bad arguments"};
        if (tree->device != ctx->device) throw Fail{GT_ERR_DEVICE, "the tree belongs to another device"};
        DeviceGuard dg(ctx->device);
        run_tree_audit(ctx, tree, n_bad, msg, msglen);
    });
}

int gt_mac_ceiling(gt_context* ctx, const gt_tree* tree, const double* amag, double alpha, int window,
                   int64_t n_windows, const int64_t* windows, int mode, double eps, double cost_exp,
                   double rho_lo, double rho_hi, int mem, double* ax, double* ay, double* az,
                   int64_t* counts) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!tree || !amag || n_windows < 0 || (n_windows > 0 && (!windows || !ax || !ay || !az || !counts)))
            throw Fail{GT_ERR_INVALID, "bad arguments"};
        if (window < 1 || window > 32) throw Fail{GT_ERR_INVALID, "window must be in [1, 32]"};
        if (mode < 0 || mode > 5) throw Fail{GT_ERR_INVALID, "mode must be in [0, 5]"};
        if (!(alpha > 0) || !(eps >= 0) || !(rho_hi >= rho_lo) || !(cost_exp >= 0.0 && cost_exp <= 4.0))
            throw Fail{GT_ERR_INVALID, "bad alpha, eps, cost exponent or band"};
        if (tree->n_systems > 1) throw Fail{GT_ERR_UNSUPPORTED, "gt_mac_ceiling takes a single-system tree"};
        if (n_windows > (int64_t)INT32_MAX / 32) throw Fail{GT_ERR_INVALID, "too many windows"};
        const int64_t nwin_all = (tree->n_live + window - 1) / window;
        if (mem == GT_MEM_HOST)
            for (int64_t k = 0; k < n_windows; ++k)
                if (windows[k] < 0 || windows[k] >= nwin_all) throw Fail{GT_ERR_INVALID, "window index out of range"};
        DeviceGuard dg(ctx->device);
        const double* da = stage_in(ctx, kSlotIn0, amag, tree->n_live, mem);
        const int64_t* dw = stage_in(ctx, kSlotIn1, windows, n_windows, mem);
        const int64_t ns = n_windows * window;
        double* ox = out_buf(ctx, kSlotOut0, ax, ns, mem);
        double* oy = out_buf(ctx, kSlotOut1, ay, ns, mem);
        double* oz = out_buf(ctx, kSlotOut2, az, ns, mem);
        int64_t* oc = out_buf(ctx, kSlotOut3, counts, n_windows * 5, mem);
        run_mac_ceiling(ctx, tree, da, alpha, window, n_windows, dw, mode, eps, cost_exp, rho_lo, rho_hi, ox, oy, oz,
                        (unsigned long long*)oc);
        copy_out(ctx, ax, (const double*)ox, ns, mem);
        copy_out(ctx, ay, (const double*)oy, ns, mem);
        copy_out(ctx, az, (const double*)oz, ns, mem);
        copy_out(ctx, counts, (const int64_t*)oc, n_windows * 5, mem);
        finish(ctx, true);
    });
}

int gt_mac_train(gt_context* ctx, int64_t n, const float* features, const float* labels,
                 const gt_mac_train_options* opt, int mem, float* model, double* loss) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (n <= 0 || !features || !labels || !model) throw Fail{GT_ERR_INVALID, "bad arguments"};
        gt_mac_train_options o;
        gt_mac_train_options_default(&o);
        if (opt) o = *opt;
        if (o.epochs < 1 || o.batch < 1 || !(o.lr > 0) || !(o.tau > 0 && o.tau < 1))
            throw Fail{GT_ERR_INVALID, "bad training options"};
        DeviceGuard dg(ctx->device);
        const float* X = stage_in(ctx, kSlotIn0, features, n * GT_MAC_FEATURES, mem);
        const float* Y = stage_in(ctx, kSlotIn1, labels, n, mem);
        run_mac_train(ctx, n, X, Y, o, model, loss);
    });
}

int gt_mac_predict(gt_context* ctx, const float* model, int64_t n, const float* features, int mem,
                   float* out) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!model || n < 0 || (n > 0 && (!features || !out))) throw Fail{GT_ERR_INVALID, "bad arguments"};
        DeviceGuard dg(ctx->device);
        const float* dm = stage_in(ctx, kSlotIn2, model, (int64_t)GT_MAC_MODEL_FLOATS, GT_MEM_HOST);
        const float* X = stage_in(ctx, kSlotIn0, features, n * GT_MAC_FEATURES, mem);
        float* o = out_buf(ctx, kSlotOut0, out, n, mem);
        run_mac_predict(ctx, dm, n, X, o);
        copy_out(ctx, out, (const float*)o, n, mem);
        finish(ctx, true);
    });
}

int gt_mac_gradient(gt_context* ctx, const float* model, int64_t n, const float* features,
                    const float* labels, double tau, int mem, float* grad, double* loss) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        check_mem(mem);
        if (!model || n <= 0 || n > (int64_t)INT32_MAX || !features || !labels || !grad)
            throw Fail{GT_ERR_INVALID, "bad arguments"};
        if (!(tau > 0 && tau < 1)) throw Fail{GT_ERR_INVALID, "tau must be in (0, 1)"};
        DeviceGuard dg(ctx->device);
        const float* dm = stage_in(ctx, kSlotIn2, model, (int64_t)GT_MAC_MODEL_FLOATS, GT_MEM_HOST);
        const float* X = stage_in(ctx, kSlotIn0, features, n * GT_MAC_FEATURES, mem);
        const float* Y = stage_in(ctx, kSlotIn1, labels, n, mem);
        float* g = out_buf(ctx, kSlotOut0, grad, (int64_t)GT_MAC_PARAM_FLOATS, mem);
        run_mac_grad(ctx, dm, X, Y, nullptr, 0, (int)n, tau, g, loss);
        copy_out(ctx, grad, (const float*)g, (int64_t)GT_MAC_PARAM_FLOATS, mem);
        finish(ctx, true);
    });
}

int gt_measure_peaks(gt_context* ctx, double* fp32_tflops, double* fp64_tflops) {
    if (!ctx) return GT_ERR_INVALID;
    return guarded(ctx, [&] {
        DeviceGuard dg(ctx->device);
        run_peaks(ctx, fp32_tflops, fp64_tflops);
    });
}

}  // extern "C"
