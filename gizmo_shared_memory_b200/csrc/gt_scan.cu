// Device-wide exclusive scan and stable LSD radix sort of (u64 key, u32 value) pairs.
//
// Both use reduce-then-scan (per-tile totals, one scan of the totals, then per-tile scans or
// scatters) rather than decoupled look-back: no block ever waits on another, so nothing can spin
// on a shared GPU.  Tiles are sized so a 16M-key pass runs as ~8k blocks, far above 148 SMs x
// resident blocks.  The sort replaces the reference's __gnu_parallel::sort of particle indices by
// key (shmem/tree.cc:420-421) and the MPI code's (key, index) merge sort (system/peano.cc:408-440);
// unlike the former it is stable, so equal keys keep particle-index order.
#include "gt_internal.cuh"

namespace gt {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the block total through *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t block_tot;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t inc = warp_incl_scan(v);
    if (lane == 31) warp_tot[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < nw ? warp_tot[lane] : 0u;
        const uint32_t wi = warp_incl_scan(w);
        if (lane < nw) warp_tot[lane] = wi - w;
        if (lane == nw - 1) block_tot = wi;
    }
    __syncthreads();
    const uint32_t res = inc - v + warp_tot[wid];
    if (total) *total = block_tot;
    __syncthreads();
    return res;
}

// n_dev (optional): the number of items, on the device, at most n (the launch is sized by n).
__global__ void tile_sum_kernel(const uint32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ sums,
                                const int64_t* __restrict__ n_dev) {
    if (n_dev) n = min(n, *n_dev);
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    uint32_t tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One block scans all tile totals in place (exclusive); total to total_out.
__global__ void scan_sums_kernel(uint32_t* __restrict__ sums, int nb, uint32_t* __restrict__ total_out,
                                 const int64_t* __restrict__ n_dev) {
    if (n_dev) nb = (int)min((int64_t)nb, (*n_dev + kScanTile - 1) / kScanTile);
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    const int lo = threadIdx.x * per, hi = min(nb, lo + per);
    uint32_t s = 0;
    for (int i = lo; i < hi; ++i) s += sums[i];
    uint32_t tot;
    uint32_t run = block_excl_scan(s, &tot);
    for (int i = lo; i < hi; ++i) {
        const uint32_t v = sums[i];
        sums[i] = run;
        run += v;
    }
    if (threadIdx.x == 0 && total_out) *total_out = tot;
}

// Blocked arrangement inside the tile: thread t owns items [t*8, t*8+8) so the scan order is the
// index order.
__global__ void tile_scan_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, int64_t n,
                                 const uint32_t* __restrict__ sums, const int64_t* __restrict__ n_dev) {
    if (n_dev) n = min(n, *n_dev);
    if ((int64_t)blockIdx.x * kScanTile >= n) return;  // the whole block lies past the items
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        s += v[k];
    }
    uint32_t run = block_excl_scan(s, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
}

// ---------------------------------------------------------------------------------------------
// Radix sort
// ---------------------------------------------------------------------------------------------

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;                            // per thread
constexpr int kSortTile = kSortThreads * kSortItems;     // 2048 keys per block
constexpr int kWarpSpan = 32 * kSortItems;               // 256 consecutive keys per warp
constexpr int kRadix = 256;

__global__ void radix_hist_kernel(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                  uint32_t* __restrict__ hist, int nblocks) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + (int64_t)k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one 8-bit digit.  Warp w owns keys [w*256, w*256+256) of the tile and walks
// them 32 at a time in index order; lanes with equal digits are ranked with __match_any_sync, so
// the destination order equals the source order within every digit.  The tile is first reordered
// by digit in shared memory, and then written out in that order: consecutive threads store
// consecutive positions of one digit's run, instead of every lane of a warp storing to its own
// digit's bucket.
__global__ void __launch_bounds__(kSortThreads)
radix_scatter_kernel(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                     uint64_t* __restrict__ kout, uint32_t* __restrict__ vout, int64_t n, int shift,
                     const uint32_t* __restrict__ offsets, int nblocks) {
    __shared__ uint32_t wh[kSortWarps][kRadix];
    __shared__ uint32_t boff[kRadix];
    __shared__ uint32_t bstart[kRadix];   // first tile position of each digit
    __shared__ uint32_t wsum[kSortWarps];
    __shared__ uint64_t tkey[kSortTile];
    __shared__ uint32_t tval[kSortTile];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < kSortWarps * kRadix; d += kSortThreads) (&wh[0][0])[d] = 0;
    boff[threadIdx.x] = offsets[(int64_t)threadIdx.x * nblocks + blockIdx.x];
    __syncthreads();
    const int64_t tile0 = (int64_t)blockIdx.x * kSortTile;
    const int64_t base = tile0 + (int64_t)w * kWarpSpan;
    const uint32_t lt = (1u << lane) - 1u;
    uint64_t key[kSortItems];
    uint32_t val[kSortItems], rnk[kSortItems];
    int dig[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + k * 32 + lane;
        const bool ok = i < n;
        key[k] = ok ? kin[i] : 0ull;
        val[k] = ok ? vin[i] : 0u;
        dig[k] = ok ? (int)((key[k] >> shift) & 0xffu) : kRadix;  // sentinel never matches a digit
        const unsigned peers = __match_any_sync(0xffffffffu, dig[k]);
        const uint32_t before = ok ? wh[w][dig[k]] : 0u;
        rnk[k] = before + __popc(peers & lt);
        __syncwarp();
        if (ok && (peers & lt) == 0) wh[w][dig[k]] = before + __popc(peers);  // lowest peer updates
        __syncwarp();
    }
    __syncthreads();
    uint32_t total = 0;  // this block's count of digit threadIdx.x
    {   // exclusive scan over warps for each digit: warp w's keys follow warps 0..w-1
        const int d = threadIdx.x;
#pragma unroll
        for (int ww = 0; ww < kSortWarps; ++ww) {
            const uint32_t c = wh[ww][d];
            wh[ww][d] = total;
            total += c;
        }
    }
    {   // exclusive scan over digits of the block's counts: where each digit's run starts in the tile
        uint32_t v = total;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += t;
        }
        if (lane == 31) wsum[w] = v;
        __syncthreads();
        uint32_t before = 0;
        for (int ww = 0; ww < w; ++ww) before += wsum[ww];
        bstart[threadIdx.x] = before + v - total;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        if (dig[k] < kRadix) {
            const uint32_t pos = bstart[dig[k]] + wh[w][dig[k]] + rnk[k];
            tkey[pos] = key[k];
            tval[pos] = val[k];
        }
    }
    __syncthreads();
    const int nvalid = n - tile0 < kSortTile ? (int)(n - tile0) : kSortTile;
    for (int j = threadIdx.x; j < nvalid; j += kSortThreads) {
        const uint64_t kk = tkey[j];
        const int d = (int)((kk >> shift) & 0xffu);
        const uint32_t pos = boff[d] + (uint32_t)j - bstart[d];
        kout[pos] = kk;
        vout[pos] = tval[j];
    }
}

}  // namespace

void scan_exclusive_u32(gt_context* ctx, const uint32_t* in, uint32_t* out, int64_t n,
                        uint32_t* total_dev, const int64_t* n_dev) {
    if (n <= 0) {
        if (total_dev) check_cuda(cudaMemsetAsync(total_dev, 0, 4, ctx->stream), "memset");
        return;
    }
    const int nb = div_up(n, kScanTile);
    uint32_t* sums = (uint32_t*)scratch(ctx, kSlotScanB, (size_t)nb * 4);
    tile_sum_kernel<<<nb, kScanThreads, 0, ctx->stream>>>(in, n, sums, n_dev);
    check_launch(ctx, "tile_sum_kernel");
    scan_sums_kernel<<<1, 1024, 0, ctx->stream>>>(sums, nb, total_dev, n_dev);
    check_launch(ctx, "scan_sums_kernel");
    tile_scan_kernel<<<nb, kScanThreads, 0, ctx->stream>>>(in, out, n, sums, n_dev);
    check_launch(ctx, "tile_scan_kernel");
}

void radix_sort_pairs(gt_context* ctx, uint64_t* keys, uint32_t* vals, int64_t n, int bits) {
    if (n <= 1) return;
    const int nb = div_up(n, kSortTile);
    uint64_t* kb = (uint64_t*)scratch(ctx, kSlotKeysB, (size_t)n * 8);
    uint32_t* vb = (uint32_t*)scratch(ctx, kSlotValsB, (size_t)n * 4);
    uint32_t* hist = (uint32_t*)scratch(ctx, kSlotHist, (size_t)kRadix * nb * 4);
    uint64_t* ka = keys;
    uint32_t* va = vals;
    const int passes = (bits + 7) / 8;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        radix_hist_kernel<<<nb, kSortThreads, 0, ctx->stream>>>(ka, n, shift, hist, nb);
        check_launch(ctx, "radix_hist_kernel");
        scan_exclusive_u32(ctx, hist, hist, (int64_t)kRadix * nb, nullptr);
        radix_scatter_kernel<<<nb, kSortThreads, 0, ctx->stream>>>(ka, va, kb, vb, n, shift, hist, nb);
        check_launch(ctx, "radix_scatter_kernel");
        uint64_t* tk = ka; ka = kb; kb = tk;
        uint32_t* tv = va; va = vb; vb = tv;
    }
    if (ka != keys) {
        check_cuda(cudaMemcpyAsync(keys, ka, (size_t)n * 8, cudaMemcpyDeviceToDevice, ctx->stream), "copy keys");
        check_cuda(cudaMemcpyAsync(vals, va, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy vals");
    }
}

}  // namespace gt
