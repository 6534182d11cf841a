/*
 * sort.cu - stable LSD radix sort of (key, value) pairs on the device, and
 * the per-tile ranges.
 *
 * Reference: radix_sort_64bit, src/raster/radix_sort.mojo:39-87 (eight
 * stable 8-bit LSD passes with 256 buckets), and
 * TileRangeIndex.build_from_sorted_keys, src/raster/binning.mojo:51-73.
 *
 * B200 design (onesweep, Adinets & Merrill 2022), for 32- or 64-bit keys:
 *  - one histogram pass reads the keys once and counts every digit that
 *    varies (the frame's tile sort needs none: the emission that writes the
 *    tile ids counts them). A digit is constant when no two keys differ in
 *    that byte (the OR of all keys and the OR of all complemented keys,
 *    gathered by the kernel that produced them, tell which); a pass over a
 *    constant digit leaves a stable sort unchanged, so it is skipped on the
 *    device.
 *  - each digit pass is one persistent kernel: a CTA takes 4096-key tiles in
 *    ticket order, counts the tile's digits and publishes the counts at
 *    once, ranks its keys with a warp-level multisplit (a shared match mask
 *    per digit; stable: warp order, then item order, then lane order)
 *    straight into shared memory, and then resolves the global
 *    digit offsets by decoupled look-back over earlier tiles. Keys are
 *    written out in digit runs.
 *  - every wait on another CTA's descriptor is bounded.
 * Per pass and pair: (sizeof key + 4) B read and written.
 *
 * Tile ranges: the frame's tile sort leaves its ids in final order in the
 * pass over the highest varying byte, which writes each tile's range from
 * the edges of the runs of equal ids in its pass tiles (atomic minimum of
 * the run starts, maximum of the run ends); a small kernel then counts the
 * touched tiles and finds each view's first instance from the ranges.
 */
#include "splat_common.cuh"

namespace lumen {

__device__ __forceinline__ unsigned int varying_digits(const SortControl* c, int nbytes) {
    const unsigned long long v = c->key_or & c->key_or_not;
    unsigned int m = 0;
    for (int d = 0; d < nbytes; ++d)
        if ((v >> (8 * d)) & 0xFFull) m |= 1u << d;
    return m;
}

__device__ __forceinline__ long long sort_count(const SortControl* c, long long capacity) {
    const long long k = (long long)c->n;
    return k < capacity ? k : capacity;
}

/* Histogram of every varying digit; clears the look-back regions of the
 * passes that will run; optionally fills the tile ranges with -1.
 *
 * Each thread counts runs of kRun consecutive keys: equal digits in a row
 * are summed in a register and added to the warp's shared histogram once
 * per run. Tile ids in emission order form long runs in their high byte
 * (the instances of one splat row), so those collapse to a few atomics;
 * random digits cost one shared atomic per key, with no warp-wide match. */
template <typename KeyT>
__global__ void __launch_bounds__(256)
histogram_kernel(const KeyT* __restrict__ keys, long long capacity, SortControl* sc, unsigned int* lb,
                 long long lb_tiles_cap, int tile_keys, int* ranges, const long long* n_range_tiles) {
    chain_begin();
    constexpr int kBytes = (int)sizeof(KeyT);
    constexpr int kRun = kBytes == 8 ? 8 : 16;           /* 64 bytes of keys per thread and run */
    /* a histogram set per warp (per pair of warps for 8-byte keys, to stay
     * within 32 KB) so warps do not contend on the same shared bins */
    constexpr int kWarps = kBytes == 8 ? 4 : 8;
    __shared__ unsigned int h[kWarps][kBytes][256];
    const int tid = threadIdx.x, warp = (tid >> 5) % kWarps;
    const long long K = sort_count(sc, capacity);
    const unsigned int varying = K > 1 ? varying_digits(sc, kBytes) : 0u;
    for (int j = tid; j < kWarps * kBytes * 256; j += 256) (&h[0][0][0])[j] = 0u;
    __syncthreads();
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    const long long gtid = (long long)blockIdx.x * blockDim.x + tid;
    const bool vec = ((uintptr_t)keys & 15u) == 0;   /* runs start 64-byte apart from the base */
    if (varying) {
        for (long long c = gtid; c * kRun < K; c += nthreads) {
            const long long i0 = c * kRun;
            KeyT k[kRun];
            const int nk = (int)(K - i0 < kRun ? K - i0 : kRun);
            if (nk == kRun && vec) {
                const uint4* src = reinterpret_cast<const uint4*>(keys + i0);
#pragma unroll
                for (int q = 0; q < kRun * kBytes / 16; ++q) {
                    const uint4 v = src[q];
                    reinterpret_cast<uint4*>(k)[q] = v;
                }
            } else {
#pragma unroll
                for (int r = 0; r < kRun; ++r) k[r] = r < nk ? keys[i0 + r] : (KeyT)0;
            }
#pragma unroll
            for (int d = 0; d < kBytes; ++d) {
                if (!(varying & (1u << d))) continue;
                unsigned int prev = (unsigned int)((k[0] >> (8 * d)) & 0xFF), run = 1;
#pragma unroll
                for (int r = 1; r < kRun; ++r) {
                    if (r >= nk) break;
                    const unsigned int b = (unsigned int)((k[r] >> (8 * d)) & 0xFF);
                    if (b == prev) {
                        ++run;
                    } else {
                        atomicAdd(&h[warp][d][prev], run);
                        prev = b;
                        run = 1;
                    }
                }
                atomicAdd(&h[warp][d][prev], run);
            }
        }
    }
    __syncthreads();
    if (varying) {
        for (int j = tid; j < kBytes * 256; j += 256) {
            const int d = j >> 8, b = j & 255;
            unsigned int c = 0;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) c += h[w][d][b];
            if ((varying & (1u << d)) && c) atomicAdd(&sc->hist[d][b], c);
        }
        const long long tiles = (K + tile_keys - 1) / tile_keys;
        for (int d = 0; d < kBytes; ++d) {
            if (!(varying & (1u << d))) continue;
            unsigned int* region = lb + (size_t)d * (size_t)lb_tiles_cap * 256;
            for (long long j = gtid; j < tiles * 256; j += nthreads) region[j] = 0u;
        }
    }
    if (ranges) {
        const long long n_range_ints = 2 * *n_range_tiles;
        for (long long j = gtid; j < n_range_ints; j += nthreads) ranges[j] = -1;
    }
    if (blockIdx.x == 0 && tid == 0) {
        sc->varying = varying;
        sc->sorted_buffer = (unsigned int)(__popc(varying) & 1);
    }
}

template <typename KeyT, int kItems>
struct PassSmem {
    KeyT keys[kSortThreads * kItems];
    unsigned int vals[kSortThreads * kItems];
    unsigned int whist[kSortThreads / 32][256];
    unsigned int match[2][kSortThreads / 32][256];   /* per item parity and warp: lanes holding each digit */
    unsigned int digit_start[256];
    long long gbase[256];
    unsigned int goffset[256];
    unsigned int warp_sums[kSortThreads / 32];
    unsigned int tile;
};

/* Sum over earlier tiles of digit t's count, walking back until a tile with
 * an inclusive prefix is found. The descriptors are read kLookbackWindow at
 * a time (independent loads, one round trip per window): when every CTA
 * starts at once, tile k's walk is about k/2 tiles long. A descriptor not
 * yet published stops the window; the walk resumes from it. Wider windows
 * measured slower (more loads per step than the walks save). */
constexpr int kLookbackWindow = 4;

__device__ __forceinline__ unsigned int lookback_digit(const unsigned int* lb, int tile, int t, unsigned int* err) {
    unsigned int excl = 0;
    int j = tile - 1;
    int spins = 0;
    while (j >= 0) {
        unsigned int d[kLookbackWindow];
#pragma unroll
        for (int w = 0; w < kLookbackWindow; ++w)
            d[w] = j - w >= 0 ? ld_volatile_u32(lb + (size_t)(j - w) * 256 + t) : 0u;
        bool done = false, stalled = false;
#pragma unroll
        for (int w = 0; w < kLookbackWindow; ++w) {
            if (done || stalled) continue;
            const unsigned int v = d[w];
            if (!(v >> 30)) {
                stalled = true;
            } else {
                excl += v & kDescMask32;
                --j;
                if ((v >> 30) == 2) done = true;
            }
        }
        if (done) break;
        if (stalled) {
            if (++spins >= kSpinLimit) {
                atomicOr(err, LUMEN_GPU_ERR_SPIN_TIMEOUT);
                break;
            }
            __nanosleep(32);
        }
    }
    return excl;
}

/* Where the tile sort's last digit pass writes the tile ranges
 * (binning.mojo:51-73), or ranges == nullptr for every other sort. The
 * ranges hold (-1, -1) before the sort. */
struct TileRangeSink {
    int* ranges;
    const long long* n_tiles;   /* the batch's tile count (ids at or above it are a bounds error) */
    unsigned int* done;         /* set to 1 by the pass that wrote the ranges */
};

/* Key j of a pass tile (nvalid keys, in sorted order in shared memory) went
 * to global position pos. A digit's keys go to consecutive positions, so a
 * run of equal ids inside the pass tile covers consecutive positions: the
 * tile's range starts at the smallest run start over all pass tiles and ends
 * after the largest run end (a range's -1 start is the largest unsigned
 * value, so the minimum replaces it). */
template <typename KeyT>
__device__ __forceinline__ void tile_range_edges(const TileRangeSink& sink, const KeyT* skeys, int j, int nvalid,
                                                 KeyT kk, long long pos, long long n_tiles, unsigned int* err) {
    const bool first = j == 0 || skeys[j - 1] != kk;
    const bool last = j + 1 == nvalid || skeys[j + 1] != kk;
    if (!first && !last) return;
    const unsigned int t = (unsigned int)kk;
    if ((long long)t >= n_tiles) {   /* self-check: a tile id outside the grid */
        atomicOr(err, LUMEN_GPU_ERR_BOUNDS);
        return;
    }
    if (first) atomicMin(reinterpret_cast<unsigned int*>(sink.ranges + 2 * (size_t)t), (unsigned int)pos);
    if (last) atomicMax(sink.ranges + 2 * (size_t)t + 1, (int)(pos + 1));
}

/* kItems keys per thread: tiles of 256 * kItems keys. */
template <typename KeyT, int kItems>
__global__ void __launch_bounds__(kSortThreads, sizeof(KeyT) == 4 ? (kItems <= 8 ? 4 : kItems <= 16 ? 3 : 2) : 2)
onesweep_pass_kernel(KeyT* k0, unsigned int* v0, KeyT* k1, unsigned int* v1, long long capacity, SortControl* sc,
                     unsigned int* lb_all, long long lb_tiles_cap, unsigned int* err, int digit, TileRangeSink sink) {
    chain_begin();
    constexpr int kTileKeys = kSortThreads * kItems;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PassSmem<KeyT, kItems>& s = *reinterpret_cast<PassSmem<KeyT, kItems>*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    /* the digits that vary, from the producer's key statistics (the same
     * rule as the histogram kernel's, for sorts whose histogram the producer
     * counted) */
    const unsigned int varying = sort_count(sc, capacity) > 1 ? varying_digits(sc, (int)sizeof(KeyT)) : 0u;
    if (blockIdx.x == 0 && tid == 0) {
        sc->varying = varying;
        sc->sorted_buffer = (unsigned int)(__popc(varying) & 1);
    }
    if (!(varying & (1u << digit))) return;
    const int src = __popc(varying & ((1u << digit) - 1u)) & 1;
    const KeyT* __restrict__ kin = src ? k1 : k0;
    const unsigned int* __restrict__ vin = src ? v1 : v0;
    KeyT* __restrict__ kout = src ? k0 : k1;
    unsigned int* __restrict__ vout = src ? v0 : v1;
    const long long K = sort_count(sc, capacity);
    const long long ntiles = (K + kTileKeys - 1) / kTileKeys;
    const int shift = 8 * digit;
    unsigned int* lb = lb_all + (size_t)digit * (size_t)lb_tiles_cap * 256;
    /* the pass over the highest varying digit leaves the ids in their final
     * order and writes the tile ranges from the run edges it sees in each
     * pass tile (32-bit tile ids only) */
    const bool emit_ranges = sizeof(KeyT) == 4 && sink.ranges != nullptr && (varying >> digit) == 1u;
    const long long n_tiles = emit_ranges ? *sink.n_tiles : 0;
    if (emit_ranges && blockIdx.x == 0 && tid == 0) *sink.done = 1u;

    /* global exclusive offsets of this digit's buckets */
    {
        const unsigned int c = sc->hist[digit][tid];
        unsigned int x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s.warp_sums[warp] = x;
        __syncthreads();
        unsigned int wb = 0;
        for (int w = 0; w < warp; ++w) wb += s.warp_sums[w];
        s.goffset[tid] = wb + x - c;
        __syncthreads();
    }

    /* the match masks start clear; each item's leaders clear what it set */
    for (int j = tid; j < 2 * (kSortThreads / 32) * 256; j += kSortThreads) (&s.match[0][0][0])[j] = 0u;

    for (;;) {
        if (tid == 0) s.tile = atomicAdd(&sc->pass_ticket[digit], 1u);
        __syncthreads();
        const long long tile = s.tile;
        if (tile >= ntiles) break;
        const long long base = tile * kTileKeys;

        /* warp w owns keys [base + w*512, +512); item i of lane l is base + w*512 + i*32 + l */
        KeyT k[kItems];
        unsigned int v[kItems];
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const long long idx = base + warp * (kItems * 32) + it * 32 + lane;
            const bool valid = idx < K;
            k[it] = valid ? kin[idx] : (KeyT)0;
            v[it] = valid ? vin[idx] : 0u;
        }
        const long long wbase = base + warp * (kItems * 32);
        for (int b = lane; b < 256; b += 32) s.whist[warp][b] = 0u;
        __syncwarp();
        /* the tile's digit counts come first (per-warp shared histograms; the
         * order of the increments does not matter), so that the tile's
         * aggregate is published before its keys are ranked and the
         * look-back chain of the tiles after it moves on sooner */
#pragma unroll
        for (int it = 0; it < kItems; ++it)
            if (wbase + it * 32 + lane < K) atomicAdd(&s.whist[warp][(unsigned int)((k[it] >> shift) & 0xFF)], 1u);
        __syncthreads();
        /* digit t: warp-exclusive offsets and the tile's count */
        const int t = tid;
        unsigned int run = 0;
#pragma unroll
        for (int w = 0; w < kSortThreads / 32; ++w) {
            const unsigned int c = s.whist[w][t];
            s.whist[w][t] = run;
            run += c;
        }
        const unsigned int count = run;
        st_volatile_u32(lb + (size_t)tile * 256 + t, (tile == 0 ? kDescIncl32 : kDescAgg32) | count);
        {
            unsigned int x = count;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) s.warp_sums[warp] = x;
            __syncthreads();
            unsigned int wb = 0;
            for (int w = 0; w < warp; ++w) wb += s.warp_sums[w];
            s.digit_start[t] = wb + x - count;
        }
        __syncthreads();
        /* warp-level stable multisplit (warp order, then item order, then
         * lane order): each lane sets its bit in the shared mask of its
         * digit, so after a warp barrier the mask names the lanes holding the
         * same digit (one shared atomic per key, where a ballot per digit bit
         * costs eight vote and select steps and a match instruction slows
         * down with the number of distinct digits). The lowest such lane
         * advances the warp's running count of the digit, which starts at its
         * warp-exclusive offset, and clears the mask; a key's rank is then its
         * place in the tile's digit run and it goes straight to its slot in
         * shared memory. Items alternate between two mask sets, so the
         * clearing of one item's masks needs no barrier of its own before the
         * next item sets the other set. */
#pragma unroll
        for (int it = 0; it < kItems; ++it) {
            const bool valid = wbase + it * 32 + lane < K;
            const unsigned int d = (unsigned int)((k[it] >> shift) & 0xFF);
            unsigned int* mk = s.match[it & 1][warp];
            if (valid) atomicOr(&mk[d], 1u << lane);
            __syncwarp();
            const unsigned int peers = valid ? mk[d] : 0u;
            unsigned int prior = 0;
            if (valid) prior = s.whist[warp][d];
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) {
                s.whist[warp][d] = prior + __popc(peers);
                mk[d] = 0u;
            }
            if (valid) {
                const unsigned int pos = s.digit_start[d] + prior + __popc(peers & lanemask_lt());
                s.keys[pos] = k[it];
                s.vals[pos] = v[it];
            }
        }
        /* the look-back runs once the keys are in shared memory (their
         * registers are free for a wide window of descriptors) */
        unsigned int excl = 0;
        if (tile > 0) {
            excl = lookback_digit(lb, (int)tile, t, err);
            st_volatile_u32(lb + (size_t)tile * 256 + t, kDescIncl32 | (excl + count));
        }
        s.gbase[t] = (long long)s.goffset[t] + (long long)excl - (long long)s.digit_start[t];
        __syncthreads();
        const int nvalid = (int)((K - base) < kTileKeys ? (K - base) : kTileKeys);
        if (nvalid == kTileKeys) {
#pragma unroll
            for (int it = 0; it < kItems; ++it) {
                const int j = it * kSortThreads + tid;
                const KeyT kk = s.keys[j];
                const unsigned int d = (unsigned int)((kk >> shift) & 0xFF);
                const long long out = s.gbase[d] + j;
                kout[out] = kk;
                vout[out] = s.vals[j];
                if (emit_ranges) tile_range_edges(sink, s.keys, j, kTileKeys, kk, out, n_tiles, err);
            }
        } else {
            for (int j = tid; j < nvalid; j += kSortThreads) {
                const KeyT kk = s.keys[j];
                const unsigned int d = (unsigned int)((kk >> shift) & 0xFF);
                const long long out = s.gbase[d] + j;
                kout[out] = kk;
                vout[out] = s.vals[j];
                if (emit_ranges) tile_range_edges(sink, s.keys, j, nvalid, kk, out, n_tiles, err);
            }
        }
        __syncthreads();
    }
}

/* When the tile sort's last digit pass wrote the ranges: the touched-tile
 * count and each view's first instance (the smallest range start among its
 * tiles; tile ids are view-major), from the 2 * n_tiles range entries. */
__device__ void ranges_epilogue(ViewTable* vt, const int* ranges, Control* ctrl) {
    const long long n_tiles = vt->hdr.total_tiles;
    const int n_views = vt->hdr.n_views;
    const int lane = threadIdx.x & 31;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    unsigned int touched = 0;
    for (long long wb = (long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); wb < n_tiles; wb += nthreads) {
        const long long t = wb + lane;
        const bool valid = t < n_tiles;
        /* an empty tile's start, -1, is the largest unsigned value */
        const unsigned int start = valid ? (unsigned int)ranges[2 * (size_t)t] : 0xFFFFFFFFu;
        touched += start != 0xFFFFFFFFu;
        const int v = !valid ? -1 : n_views > 1 ? find_view_by_tile(vt, n_views, t) : 0;
        const int v0 = __shfl_sync(0xffffffffu, v, 0);
        if (__all_sync(0xffffffffu, v == v0 || v < 0)) {
            const unsigned int m = __reduce_min_sync(0xffffffffu, start);
            if (lane == 0 && m != 0xFFFFFFFFu)
                atomicMin(reinterpret_cast<unsigned long long*>(&vt->view[v0].inst_begin), (unsigned long long)m);
        } else if (start != 0xFFFFFFFFu) {
            atomicMin(reinterpret_cast<unsigned long long*>(&vt->view[v].inst_begin), (unsigned long long)start);
        }
    }
    touched = __reduce_add_sync(0xffffffffu, touched);
    if (lane == 0 && touched) atomicAdd(&ctrl->touched_tiles, touched);
}

/* binning.mojo:51-73 in parallel, on tile-sorted 32-bit tile ids: a tile's
 * range starts where its id first appears and ends after it last appears.
 * Empty tiles keep the (-1, -1) written before the sort. When a tile-id byte
 * varies, the tile sort's last digit pass has written the ranges and this
 * kernel only finishes them (ranges_epilogue); otherwise it reads the ids:
 *
 * Each lane takes 8 consecutive ids per round (two 16-byte loads; the
 * frame's key buffers are 16-byte aligned) and its neighbours' ids come
 * from the adjacent lanes. The ids are sorted, so when the id before the
 * group equals the id after it, all eight equal it and the group holds no
 * boundary: one comparison for almost every group. */
constexpr int kRangeIds = 8;

__global__ void __launch_bounds__(256)
tile_ranges_kernel(const unsigned int* k0, const unsigned int* k1, long long capacity, ViewTable* vt,
                   int* ranges, Control* ctrl) {
    chain_begin();
    if (ctrl->ranges_by_sort) {
        ranges_epilogue(vt, ranges, ctrl);
        return;
    }
    const SortControl* sc = &ctrl->tile_sort;
    const long long n_tiles = vt->hdr.total_tiles;
    const int n_views = vt->hdr.n_views;
    const long long K = sort_count(sc, capacity);
    const unsigned int* __restrict__ keys = sc->sorted_buffer ? k1 : k0;
    const int lane = threadIdx.x & 31;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    unsigned int touched = 0;
    /* the warp's first id, so that the loop and its shuffles are warp-uniform */
    for (long long wb = ((long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31)) * kRangeIds; wb < K;
         wb += nthreads * kRangeIds) {
        const long long i0 = wb + kRangeIds * lane;
        unsigned int k[kRangeIds];
        if (i0 + kRangeIds - 1 < K) {
            const uint4 q0 = *reinterpret_cast<const uint4*>(keys + i0);
            const uint4 q1 = *reinterpret_cast<const uint4*>(keys + i0 + 4);
            k[0] = q0.x; k[1] = q0.y; k[2] = q0.z; k[3] = q0.w;
            k[4] = q1.x; k[5] = q1.y; k[6] = q1.z; k[7] = q1.w;
        } else {
#pragma unroll
            for (int r = 0; r < kRangeIds; ++r) k[r] = i0 + r < K ? keys[i0 + r] : 0xFFFFFFFFu;
        }
        const unsigned int up = __shfl_up_sync(0xffffffffu, k[kRangeIds - 1], 1);
        const unsigned int down = __shfl_down_sync(0xffffffffu, k[0], 1);
        if (i0 >= K) continue;
        const unsigned int prev = lane > 0 ? up : (i0 > 0 ? keys[i0 - 1] : 0xFFFFFFFFu);
        const unsigned int next = lane < 31 ? down : (i0 + kRangeIds < K ? keys[i0 + kRangeIds] : 0xFFFFFFFFu);
        if (i0 > 0 && i0 + kRangeIds < K && prev == next && (long long)next < n_tiles) continue;
#pragma unroll
        for (int r = 0; r < kRangeIds; ++r) {
            const long long i = i0 + r;
            if (i >= K) break;
            const unsigned int t = k[r];
            if ((long long)t >= n_tiles) {   /* self-check: a tile id outside the grid */
                atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
                continue;
            }
            const unsigned int before = r == 0 ? prev : k[r - 1];
            const unsigned int after = r == kRangeIds - 1 ? next : k[r + 1];   /* 0xFFFFFFFF past the end */
            if (i == 0 || before != t) {
                ranges[2 * (size_t)t] = (int)i;
                ++touched;
                /* the first instance of a view (tile ids are view-major) */
                const int v = find_view_by_tile(vt, n_views, t);
                if (i == 0 || (long long)before < vt->view[v].tile_begin) vt->view[v].inst_begin = i;
            }
            if (i == K - 1 || after != t) ranges[2 * (size_t)t + 1] = (int)(i + 1);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) touched += __shfl_xor_sync(0xffffffffu, touched, o);
    if (lane == 0 && touched) atomicAdd(&ctrl->touched_tiles, touched);
}

/* OR and OR-of-complement of n keys and the pair count, for sorts whose
 * keys come from the caller (lumen_gpu_sort_pairs). */
template <typename KeyT>
__global__ void __launch_bounds__(256)
key_stats_kernel(const KeyT* __restrict__ keys, long long n, SortControl* sc) {
    unsigned long long o = 0ull, no = 0ull;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += nthreads) {
        const unsigned long long k = (unsigned long long)keys[i];
        o |= k;
        no |= ~k;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        o |= __shfl_xor_sync(0xffffffffu, o, off);
        no |= __shfl_xor_sync(0xffffffffu, no, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicOr(&sc->key_or, o);
        atomicOr(&sc->key_or_not, no);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->n = (unsigned long long)n;
}

/* Rebuild the reference's 64-bit keys: (tile << 32) | depth key of the
 * instance's splat. */
__global__ void sorted_keys64_kernel(const unsigned int* k0, const unsigned int* k1, const unsigned int* v0,
                                     const unsigned int* v1, const LumenSplatRecord* records, long long capacity,
                                     int key_mode, const Control* ctrl, unsigned long long* out) {
    const SortControl* sc = &ctrl->tile_sort;
    const long long K = sort_count(sc, capacity);
    const unsigned int* keys = sc->sorted_buffer ? k1 : k0;
    const unsigned int* vals = sc->sorted_buffer ? v1 : v0;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < K; i += nthreads) {
        const unsigned int v = vals[i];
        out[i] = ((unsigned long long)keys[i] << 32) | depth_key(records[v].depth, key_mode);
    }
}

/* key_bytes: the low bytes that can vary at all (a pass per byte is
 * launched; among those, passes over bytes that turn out constant exit at
 * once). */
template <typename KeyT, int kItems>
void launch_sort_impl(KeyT* k0, unsigned int* v0, KeyT* k1, unsigned int* v1, long long capacity, SortControl* sc,
                      unsigned int* lb, long long lb_tiles_cap, int* ranges, const long long* n_range_tiles,
                      unsigned int* err, int key_bytes, int num_sms, cudaStream_t st, bool counted = false,
                      TileRangeSink sink = TileRangeSink{}) {
    if (!counted)
        launch_chained(histogram_kernel<KeyT>, dim3(num_sms * 4), dim3(256), 0, st, (const KeyT*)k0, capacity, sc, lb,
                       lb_tiles_cap, kSortThreads * kItems, ranges, n_range_tiles);
    const size_t smem = sizeof(PassSmem<KeyT, kItems>);
    /* matches __launch_bounds__: all CTAs resident */
    const int ctas_per_sm = sizeof(KeyT) == 4 ? (kItems <= 8 ? 4 : kItems <= 16 ? 3 : 2) : 2;
    const int nd = key_bytes < (int)sizeof(KeyT) ? key_bytes : (int)sizeof(KeyT);
    for (int d = 0; d < nd; ++d)
        launch_chained(onesweep_pass_kernel<KeyT, kItems>, dim3(num_sms * ctas_per_sm), dim3(kSortThreads), smem, st,
                       k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, err, d, sink);
}

/* items: keys per thread of a digit pass, 8, 16 or 24 (tiles of 2048, 4096
 * or 6144 keys); lb_tiles_cap must hold ceil(capacity / (256 * items))
 * tiles. */
void launch_sort32(unsigned int* k0, unsigned int* v0, unsigned int* k1, unsigned int* v1, long long capacity,
                   SortControl* sc, unsigned int* lb, long long lb_tiles_cap, int* ranges,
                   const long long* n_range_tiles, unsigned int* err, int items, int key_bytes, int num_sms,
                   cudaStream_t st) {
    if (items == 8)
        launch_sort_impl<unsigned int, 8>(k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, ranges, n_range_tiles, err,
                                          key_bytes, num_sms, st);
    else if (items == 24)
        launch_sort_impl<unsigned int, 24>(k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, ranges, n_range_tiles,
                                           err, key_bytes, num_sms, st);
    else
        launch_sort_impl<unsigned int, 16>(k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, ranges, n_range_tiles,
                                           err, key_bytes, num_sms, st);
}

/* The frame's tile sort when the emission has counted the digit values,
 * cleared the look-back tiles and filled the ranges with -1: the digit
 * passes only, the last of which writes the tile ranges. */
void launch_tile_sort_counted(unsigned int* k0, unsigned int* v0, unsigned int* k1, unsigned int* v1,
                              long long capacity, Control* ctrl, ViewTable* vt, int* ranges, unsigned int* lb,
                              long long lb_tiles_cap, int items, int key_bytes, int num_sms, cudaStream_t st) {
    SortControl* sc = &ctrl->tile_sort;
    unsigned int* err = &ctrl->error_flags;
    const TileRangeSink sink{ranges, &vt->hdr.total_tiles, &ctrl->ranges_by_sort};
    if (items == 8)
        launch_sort_impl<unsigned int, 8>(k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, nullptr, nullptr, err,
                                          key_bytes, num_sms, st, true, sink);
    else if (items == 24)
        launch_sort_impl<unsigned int, 24>(k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, nullptr, nullptr, err,
                                           key_bytes, num_sms, st, true, sink);
    else
        launch_sort_impl<unsigned int, 16>(k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, nullptr, nullptr, err,
                                           key_bytes, num_sms, st, true, sink);
}

void launch_sort64(unsigned long long* k0, unsigned int* v0, unsigned long long* k1, unsigned int* v1,
                   long long capacity, SortControl* sc, unsigned int* lb, long long lb_tiles_cap, unsigned int* err,
                   int num_sms, cudaStream_t st) {
    launch_sort_impl<unsigned long long, kSort64Items>(k0, v0, k1, v1, capacity, sc, lb, lb_tiles_cap, nullptr,
                                                       nullptr, err, 8, num_sms, st);
}

void launch_ranges(const LumenGpuFrame& f, Control* ctrl, ViewTable* vt, int num_sms, cudaStream_t st) {
    /* the tile sort's last digit pass writes the ranges whenever a tile-id
     * byte varies, and this launch then reads only the ranges (2 * n_tiles
     * ints); otherwise (every id equal, or none) the ids are one run, which
     * a grid-stride loop over num_sms * 2 CTAs reads in a few rounds */
    const long long grid = (long long)num_sms * 2;
    launch_chained(tile_ranges_kernel, dim3((unsigned int)grid), dim3(256), 0, st, (const unsigned int*)f.keys[0],
                   (const unsigned int*)f.keys[1], (long long)f.instance_capacity, vt, f.ranges, ctrl);
}

void launch_key_stats64(const unsigned long long* keys, long long n, SortControl* sc, int num_sms, cudaStream_t st) {
    key_stats_kernel<unsigned long long><<<num_sms * 2, 256, 0, st>>>(keys, n, sc);
}

void launch_key_stats32(const unsigned int* keys, long long n, SortControl* sc, int num_sms, cudaStream_t st) {
    key_stats_kernel<unsigned int><<<num_sms * 2, 256, 0, st>>>(keys, n, sc);
}

void launch_sorted_keys64(const LumenGpuFrame& f, const Control* ctrl, int key_mode, unsigned long long* out,
                          int num_sms, cudaStream_t st) {
    sorted_keys64_kernel<<<num_sms * 4, 256, 0, st>>>(f.keys[0], f.keys[1], f.vals[0], f.vals[1], f.records,
                                                      (long long)f.instance_capacity, key_mode, ctrl, out);
}

void configure_sort_kernels() {
    cudaFuncSetAttribute(onesweep_pass_kernel<unsigned int, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(PassSmem<unsigned int, 8>));
    cudaFuncSetAttribute(onesweep_pass_kernel<unsigned int, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(PassSmem<unsigned int, 16>));
    cudaFuncSetAttribute(onesweep_pass_kernel<unsigned int, 24>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(PassSmem<unsigned int, 24>));
    cudaFuncSetAttribute(onesweep_pass_kernel<unsigned long long, kSort64Items>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(PassSmem<unsigned long long, kSort64Items>));
}

}  // namespace lumen
