/*
 * sort.cu - K3/K4: stable LSD radix sort of the (tile << 32 | depth) keys
 * with their visible-index values, and the per-tile ranges.
 *
 * Reference: radix_sort_64bit, src/raster/radix_sort.mojo:39-87 (eight
 * stable 8-bit LSD passes with 256 buckets), and
 * TileRangeIndex.build_from_sorted_keys, src/raster/binning.mojo:51-73.
 *
 * B200 design (onesweep, Adinets & Merrill 2022):
 *  - one histogram pass reads the keys once and counts every digit that
 *    varies; a digit is constant when no key differs in that byte (the OR of
 *    all keys and the OR of all complemented keys, gathered during emission,
 *    tell which). Constant digits leave a stable sort unchanged, so their
 *    passes are skipped on the device; at 1080p with millimetre keys only 4
 *    of the 8 bytes vary.
 *  - each digit pass is one persistent kernel: a CTA takes 4096-key tiles in
 *    ticket order, ranks its keys with warp-level match_any multisplit over
 *    per-warp shared-memory histograms (stable: warp order, then item order,
 *    then lane order), publishes per-digit tile counts, and resolves global
 *    digit offsets by decoupled look-back over earlier tiles. Keys are
 *    reordered in shared memory and written out in digit runs (coalesced).
 *  - every wait on another CTA's descriptor is bounded.
 * Per pass and key: 12 B read + 12 B written.
 */
#include "splat_common.cuh"

namespace lumen {

__device__ __forceinline__ unsigned int varying_from(const Control* c) {
    unsigned long long v = c->key_or & c->key_or_not;
    unsigned int m = 0;
#pragma unroll
    for (int d = 0; d < 8; ++d)
        if ((v >> (8 * d)) & 0xFFull) m |= 1u << d;
    return m;
}

__device__ __forceinline__ long long effective_count(const Control* c, long long capacity) {
    long long k = (long long)c->n_instances;
    return k < capacity ? k : capacity;
}

/* Histogram of every varying digit; also clears the look-back regions the
 * digit passes will use and fills the tile ranges with -1. */
__global__ void __launch_bounds__(256)
sort_histogram_kernel(const unsigned long long* __restrict__ keys, long long capacity, Control* ctrl,
                      unsigned int* sort_lb, long long lb_tiles_cap, int* ranges, long long n_range_ints) {
    __shared__ unsigned int h[8][256];
    const int tid = threadIdx.x, lane = tid & 31;
    const long long K = effective_count(ctrl, capacity);
    unsigned int varying = K > 1 ? varying_from(ctrl) : 0u;
    for (int j = tid; j < 8 * 256; j += 256) (&h[0][0])[j] = 0u;
    __syncthreads();
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    const long long gtid = (long long)blockIdx.x * blockDim.x + tid;
    if (varying) {
        /* warps iterate in lockstep so match_any sees full warps */
        const long long warp_base = gtid - lane;
        for (long long base = warp_base; base < K; base += nthreads) {
            const long long i = base + lane;
            const bool valid = i < K;
            const unsigned long long k = valid ? keys[i] : 0ull;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                if (!(varying & (1u << d))) continue;
                const unsigned int b = valid ? (unsigned int)((k >> (8 * d)) & 0xFF) : (0x100u + lane);
                const unsigned int peers = __match_any_sync(0xffffffffu, b);
                if (valid && lane == __ffs(peers) - 1) atomicAdd(&h[d][b], (unsigned int)__popc(peers));
            }
        }
    }
    __syncthreads();
    if (varying) {
        for (int j = tid; j < 8 * 256; j += 256) {
            const int d = j >> 8;
            const unsigned int c = (&h[0][0])[j];
            if ((varying & (1u << d)) && c) atomicAdd(&ctrl->hist[d][j & 255], c);
        }
        const long long tiles = (K + kSortTile - 1) / kSortTile;
        for (int d = 0; d < 8; ++d) {
            if (!(varying & (1u << d))) continue;
            unsigned int* region = sort_lb + (size_t)d * (size_t)lb_tiles_cap * 256;
            for (long long j = gtid; j < tiles * 256; j += nthreads) region[j] = 0u;
        }
    }
    if (ranges)
        for (long long j = gtid; j < n_range_ints; j += nthreads) ranges[j] = -1;
    if (blockIdx.x == 0 && tid == 0) {
        ctrl->varying_digits = varying;
        ctrl->sorted_buffer = (unsigned int)(__popc(varying) & 1);
    }
}

struct PassSmem {
    unsigned long long keys[kSortTile];
    unsigned int vals[kSortTile];
    unsigned int whist[kSortThreads / 32][256];
    unsigned int digit_start[256];
    long long gbase[256];
    unsigned int goffset[256];
    unsigned int warp_sums[kSortThreads / 32];
    unsigned int tile;
};

/* Sum over earlier tiles of digit `t`'s count, by walking back until a tile
 * with an inclusive prefix is found. */
__device__ __forceinline__ unsigned int lookback_digit(const unsigned int* lb, int tile, int t, unsigned int* err) {
    unsigned int excl = 0;
    for (int j = tile - 1; j >= 0; --j) {
        unsigned int v = 0;
        int spins = 0;
        for (;;) {
            v = ld_volatile_u32(lb + (size_t)j * 256 + t);
            if (v >> 30) break;
            if (++spins >= kSpinLimit) {
                atomicOr(err, LUMEN_GPU_ERR_SPIN_TIMEOUT);
                v = kDescIncl32;
                break;
            }
            __nanosleep(32);
        }
        excl += v & kDescMask32;
        if ((v >> 30) == 2) break;
    }
    return excl;
}

__global__ void __launch_bounds__(kSortThreads)
onesweep_pass_kernel(LumenGpuFrame f, long long capacity, Control* ctrl, unsigned int* sort_lb,
                     long long lb_tiles_cap, int digit) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    PassSmem& s = *reinterpret_cast<PassSmem*>(smem_raw);
    const unsigned int varying = ctrl->varying_digits;
    if (!(varying & (1u << digit))) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int src = __popc(varying & ((1u << digit) - 1u)) & 1;
    const unsigned long long* __restrict__ kin = reinterpret_cast<const unsigned long long*>(src ? f.keys[1] : f.keys[0]);
    const unsigned int* __restrict__ vin = src ? f.vals[1] : f.vals[0];
    unsigned long long* __restrict__ kout = reinterpret_cast<unsigned long long*>(src ? f.keys[0] : f.keys[1]);
    unsigned int* __restrict__ vout = src ? f.vals[0] : f.vals[1];
    const long long K = effective_count(ctrl, capacity);
    const long long ntiles = (K + kSortTile - 1) / kSortTile;
    const int shift = 8 * digit;
    unsigned int* lb = sort_lb + (size_t)digit * (size_t)lb_tiles_cap * 256;

    /* global exclusive offsets of this digit's buckets */
    {
        const unsigned int c = ctrl->hist[digit][tid];
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

    for (;;) {
        if (tid == 0) s.tile = atomicAdd(&ctrl->pass_ticket[digit], 1u);
        __syncthreads();
        const long long tile = s.tile;
        if (tile >= ntiles) break;
        const long long base = tile * kSortTile;

        /* load: warp w owns keys [base + w*512, +512), item i of lane l is base + w*512 + i*32 + l */
        unsigned long long k[kSortItems];
        unsigned int v[kSortItems];
        unsigned int dig[kSortItems];
        unsigned short rank[kSortItems];
#pragma unroll
        for (int it = 0; it < kSortItems; ++it) {
            const long long idx = base + warp * (kSortItems * 32) + it * 32 + lane;
            const bool valid = idx < K;
            k[it] = valid ? kin[idx] : 0ull;
            v[it] = valid ? vin[idx] : 0u;
            dig[it] = valid ? (unsigned int)((k[it] >> shift) & 0xFF) : (0x100u + lane);
        }
        for (int b = lane; b < 256; b += 32) s.whist[warp][b] = 0u;
        __syncwarp();
        /* warp-level stable multisplit */
#pragma unroll
        for (int it = 0; it < kSortItems; ++it) {
            const unsigned int d = dig[it];
            const unsigned int peers = __match_any_sync(0xffffffffu, d);
            const bool valid = d < 256u;
            unsigned int prior = 0;
            if (valid) prior = s.whist[warp][d];
            __syncwarp();
            if (valid && lane == __ffs(peers) - 1) s.whist[warp][d] = prior + __popc(peers);
            __syncwarp();
            rank[it] = (unsigned short)(prior + __popc(peers & lanemask_lt()));
        }
        __syncthreads();
        /* per digit t: warp-exclusive offsets and the tile's count */
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
        /* block exclusive scan of the digit counts */
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
        unsigned int excl = 0;
        if (tile > 0) {
            excl = lookback_digit(lb, (int)tile, t, &ctrl->error_flags);
            st_volatile_u32(lb + (size_t)tile * 256 + t, kDescIncl32 | (excl + count));
        }
        s.gbase[t] = (long long)s.goffset[t] + (long long)excl - (long long)s.digit_start[t];
        __syncthreads();
        /* reorder through shared memory */
#pragma unroll
        for (int it = 0; it < kSortItems; ++it) {
            const unsigned int d = dig[it];
            if (d < 256u) {
                const unsigned int pos = s.digit_start[d] + s.whist[warp][d] + rank[it];
                s.keys[pos] = k[it];
                s.vals[pos] = v[it];
            }
        }
        __syncthreads();
        const int nvalid = (int)((K - base) < kSortTile ? (K - base) : kSortTile);
        for (int j = tid; j < nvalid; j += kSortThreads) {
            const unsigned long long kk = s.keys[j];
            const unsigned int d = (unsigned int)((kk >> shift) & 0xFF);
            const long long out = s.gbase[d] + j;
            kout[out] = kk;
            vout[out] = s.vals[j];
        }
        __syncthreads();
    }
}

/* binning.mojo:51-73 in parallel: a tile's range starts where its id first
 * appears in the sorted keys and ends after it last appears. Ranges were
 * filled with -1 by the histogram kernel (empty tiles stay (-1, -1)). */
__global__ void __launch_bounds__(256)
tile_ranges_kernel(LumenGpuFrame f, long long capacity, long long n_tiles, Control* ctrl) {
    const long long K = effective_count(ctrl, capacity);
    const unsigned long long* __restrict__ keys = reinterpret_cast<const unsigned long long*>(ctrl->sorted_buffer ? f.keys[1] : f.keys[0]);
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    unsigned int touched = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < K; i += nthreads) {
        const unsigned int t = (unsigned int)(keys[i] >> 32);
        if ((long long)t >= n_tiles) {   /* self-check: a tile id outside the grid */
            atomicOr(&ctrl->error_flags, LUMEN_GPU_ERR_BOUNDS);
            continue;
        }
        const bool first = i == 0 || (unsigned int)(keys[i - 1] >> 32) != t;
        const bool last = i == K - 1 || (unsigned int)(keys[i + 1] >> 32) != t;
        if (first) { f.ranges[2 * (size_t)t] = (int)i; ++touched; }
        if (last) f.ranges[2 * (size_t)t + 1] = (int)(i + 1);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) touched += __shfl_xor_sync(0xffffffffu, touched, o);
    if ((threadIdx.x & 31) == 0 && touched) atomicAdd(&ctrl->touched_tiles, touched);
}

size_t onesweep_smem_bytes() { return sizeof(PassSmem); }

void launch_sort(LumenGpuFrame& f, Control* ctrl, unsigned int* sort_lb, long long lb_tiles_cap,
                 long long n_range_ints, int num_sms, cudaStream_t st) {
    const long long cap = (long long)f.instance_capacity;
    sort_histogram_kernel<<<num_sms * 4, 256, 0, st>>>(reinterpret_cast<const unsigned long long*>(f.keys[0]), cap, ctrl, sort_lb, lb_tiles_cap, f.ranges,
                                                       n_range_ints);
    const size_t smem = sizeof(PassSmem);
    for (int d = 0; d < 8; ++d)
        onesweep_pass_kernel<<<num_sms * 2, kSortThreads, smem, st>>>(f, cap, ctrl, sort_lb, lb_tiles_cap, d);
}

void launch_ranges(LumenGpuFrame& f, Control* ctrl, long long n_tiles, int num_sms, cudaStream_t st) {
    tile_ranges_kernel<<<num_sms * 4, 256, 0, st>>>(f, (long long)f.instance_capacity, n_tiles, ctrl);
}

/* OR and OR-of-complement of n keys, for a sort whose keys were not emitted
 * by project_emit (lumen_gpu_sort_pairs). */
__global__ void __launch_bounds__(256)
key_stats_kernel(const unsigned long long* __restrict__ keys, long long n, Control* ctrl) {
    unsigned long long o = 0ull, no = 0ull;
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += nthreads) {
        const unsigned long long k = keys[i];
        o |= k;
        no |= ~k;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        o |= __shfl_xor_sync(0xffffffffu, o, off);
        no |= __shfl_xor_sync(0xffffffffu, no, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicOr(&ctrl->key_or, o);
        atomicOr(&ctrl->key_or_not, no);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->n_instances = (unsigned long long)n;
}

void launch_key_stats(const unsigned long long* keys, long long n, Control* ctrl, int num_sms, cudaStream_t st) {
    key_stats_kernel<<<num_sms * 2, 256, 0, st>>>(keys, n, ctrl);
}

void configure_sort_kernels() {
    cudaFuncSetAttribute(onesweep_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(PassSmem));
}

}  // namespace lumen
