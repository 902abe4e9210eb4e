// exg_kernels.cu -- CUDA kernels of the B200 MPM step (sm_100a).
//
// One step is four kernel groups:
//   K1 cell-key binning sort  (replaces AMReX Redistribute)
//   K2 tile P2G               (deposit_onto_grid_momentum, deterministic fixed-point scatter)
//   K3 nodal update           (normalise, backup, time update, wall/UDF/level-set BCs, store delta)
//   K4 fused G2P              (interpolate_from_grid + moveParticles + updateVolume + apply_constitutive_model)
// plus single-thread bookkeeping kernels that keep dt, time and the
// reductions on the device so that a whole step can be replayed from a CUDA
// graph without a host round trip.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <type_traits>
#include "exg_internal.h"

// This file is compiled twice: with EXG_R_FP64 (FP64 kernels plus the
// precision-independent ones) and without (the FP32 kernels of the mixed
// path), so the two halves build in parallel.
#if defined(EXG_R_FP64)
#define EXG_R double
#define EXG_SFX(name) name##_fp64
#else
#define EXG_R float
#define EXG_SFX(name) name##_fp32
#endif

namespace exg {

namespace {
__constant__ SplineTables c_tables;
}

void EXG_SFX(upload_tables)() {
    // Coefficient tables of Source/interpolants.H:32-183 (see exg_common.cuh).
    static const SplineTables t = {
        // cubic value
        {{{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
         {{kOneBySix, 1.0, 2.0, kFourByThree}, {-kOneBySix, 0.0, 1.0, 1.0}, {kOneBySix, 0.0, -1.0, 1.0},
          {-kOneBySix, 1.0, -2.0, kFourByThree}},
         {{0.0, 0.0, 0.0, 0.0}, {-kOneByThree, -1.0, 0.0, kTwoByThree}, {0.5, -1.0, 0.0, kTwoByThree},
          {-kOneBySix, 1.0, -2.0, kFourByThree}},
         {{kOneBySix, 1.0, 2.0, kFourByThree}, {-0.5, -1.0, 0.0, kTwoByThree}, {0.5, -1.0, 0.0, kTwoByThree},
          {-kOneBySix, 1.0, -2.0, kFourByThree}},
         {{kOneBySix, 1.0, 2.0, kFourByThree}, {-0.5, -1.0, 0.0, kTwoByThree}, {kOneByThree, -1.0, 0.0, kTwoByThree},
          {0.0, 0.0, 0.0, 0.0}}},
        // cubic derivative
        {{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
         {{0.5, 2.0, 2.0}, {-0.5, 0.0, 1.0}, {0.5, 0.0, -1.0}, {-0.5, 2.0, -2.0}},
         {{0, 0, 0}, {-1.0, -2.0, 0.0}, {1.5, -2.0, 0.0}, {-0.5, 2.0, -2.0}},
         {{0.5, 2.0, 2.0}, {-1.5, -2.0, 0.0}, {1.5, -2.0, 0.0}, {-0.5, 2.0, -2.0}},
         {{0.5, 2.0, 2.0}, {-1.5, -2.0, 0.0}, {1.0, -2.0, 0.0}, {0, 0, 0}}},
        // quadratic value
        {{{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
         {{kTwoByThree, 2.0, 1.5}, {-kFourByThree, 0.0, 1.0}, {-kFourByThree, 0.0, 1.0}, {kTwoByThree, -2.0, 1.5}},
         {{4.0 / 3.0, 8.0 / 3.0, 4.0 / 3.0}, {-7.0 / 6.0, 1.0 / 6.0, 17.0 / 24.0}, {0.5, -1.5, 1.125}, {0, 0, 0}},
         {{0.5, 1.5, 1.125}, {-1.0, 0.0, 0.75}, {0.5, -1.5, 1.125}, {0, 0, 0}},
         {{0.5, 1.5, 1.125}, {-7.0 / 6.0, -1.0 / 6.0, 17.0 / 24.0}, {4.0 / 3.0, -8.0 / 3.0, 4.0 / 3.0}, {0, 0, 0}}},
        // quadratic derivative
        {{{0, 0}, {0, 0}, {0, 0}, {0, 0}},
         {{4.0 / 3.0, 2.0}, {-8.0 / 3.0, 0.0}, {-8.0 / 3.0, 0.0}, {4.0 / 3.0, -2.0}},
         {{8.0 / 3.0, 8.0 / 3.0}, {-14.0 / 6.0, 1.0 / 6.0}, {1.0, -1.5}, {0, 0}},
         {{2.0 / 2.0, 3.0 / 2.0}, {-2.0, 0.0}, {2.0 / 2.0, -3.0 / 2.0}, {0, 0}},
         {{1.0, 1.5}, {-14.0 / 6.0, -1.0 / 6.0}, {8.0 / 3.0, -8.0 / 3.0}, {0, 0}}},
        // quadratic half-interval map
        {{-1, -1, -1, -1, -1, -1}, {0, 0, 1, 2, 3, 3}, {0, 1, 1, 2, 2, -1}, {0, 0, 1, 1, 2, 2}, {0, 0, 1, 1, 2, -1}}};
    EXG_CUDA_OK(cudaMemcpyToSymbol(c_tables, &t, sizeof(t)));
}

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ void load_tables(SplineTables *dst) {
    const int n = sizeof(SplineTables) / 4;
    const int *src = reinterpret_cast<const int *>(&c_tables);
    int *d = reinterpret_cast<int *>(dst);
    for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = src[i];
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// Block-wide exclusive scan of one int per thread (blockDim.x <= 1024).
[[maybe_unused]] __device__ int block_exclusive_scan(int v, int *total, int *sh /* >= 33 ints */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        int n = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += n;
    }
    if (lane == 31) sh[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int nw = (blockDim.x + 31) >> 5;
        int s = lane < nw ? sh[lane] : 0;
        int si = s;
        for (int o = 1; o < 32; o <<= 1) {
            int n = __shfl_up_sync(0xffffffffu, si, o);
            if (lane >= o) si += n;
        }
        sh[lane] = si - s;
        if (lane == 31) sh[32] = si;
    }
    __syncthreads();
    int res = inc - v + sh[wid];
    *total = sh[32];
    __syncthreads();
    return res;
}

__device__ __forceinline__ void tile_coords(const Params &P, int t, int tc[3]) {
    tc[0] = t % P.ntile[0];
    int r = t / P.ntile[0];
    tc[1] = r % P.ntile[1];
    tc[2] = r / P.ntile[1];
}

#if defined(EXG_R_FP64)
// ---------------------------------------------------------------- K1 sort
// Cell key per particle, with the periodic wrap of Redistribute.  Keys are
// tile-major: (tile index << 3 log2 T) | (cell inside tile), so one tile's
// particles are contiguous after a stable sort by key.  With quadratic
// B-splines the key's "cell" is the nearest-node bin (dual_bin): particles
// of one bin share a 3x3x3 node window.  Particles outside the domain's
// cells are dropped either way.
// (every lane of a warp calls it: the tile histogram is warp-aggregated)
__device__ __forceinline__ void keys_body(const Params &P, double *x0, double *x1, double *x2, long long n,
                                          uint32_t *key, int *tile_count, Ctl *ctl, int wrap, long long i) {
    int t = -1;
    if (i < n) {
        double x[3] = {x0[i], x1[i], x2[i]};
        if (wrap) {
            double *xs[3] = {x0, x1, x2};
            for (int d = 0; d < 3; ++d) {
                if (!P.periodic[d]) continue;
                double L = P.phi[d] - P.plo[d];
                double y = x[d];
                if (y >= P.phi[d])
                    y -= L;
                else if (y < P.plo[d])
                    y += L;
                if (y != x[d]) {
                    x[d] = y;
                    xs[d][i] = y;
                }
            }
        }
        int iv[3];
        cell_of(P, x, iv);
        bool in = true;
        for (int d = 0; d < 3; ++d) in = in && iv[d] >= 0 && iv[d] < P.nc[d];
        if (!in) {
            key[i] = 0xFFFFFFFFu;
            atomicAdd(&ctl->lost, 1ull);
        } else {
            if (P.dual)
                for (int d = 0; d < 3; ++d) iv[d] = dual_bin(P, d, x[d]);
            const int ts = P.tshift, m = P.T - 1;
            t = ((iv[2] >> ts) * P.ntile[1] + (iv[1] >> ts)) * P.ntile[0] + (iv[0] >> ts);
            uint32_t loc = (uint32_t)((((iv[2] & m) << ts) | (iv[1] & m)) << ts | (iv[0] & m));
            key[i] = ((uint32_t)t << (3 * ts)) | loc;
        }
    }
    // warp-aggregated tile histogram (particles arrive nearly sorted, so a
    // warp's lanes usually share one tile: then one lane adds for all)
    unsigned act = __ballot_sync(0xffffffffu, t >= 0);
    const int t0 = __shfl_sync(0xffffffffu, t, 0);
    if (act == 0xffffffffu && __all_sync(0xffffffffu, t == t0)) {
        if ((threadIdx.x & 31) == 0) atomicAdd(&tile_count[t0], 32);
        return;
    }
    if (t >= 0) {
        unsigned peers = __match_any_sync(act, t);
        int leader = __ffs(peers) - 1;
        if ((int)(threadIdx.x & 31) == leader) atomicAdd(&tile_count[t], __popc(peers));
    }
}
__global__ void k_keys(Params P, double *x0, double *x1, double *x2, long long n, uint32_t *key, int *tile_count,
                       Ctl *ctl, int wrap) {
    keys_body(P, x0, x1, x2, n, key, tile_count, ctl, wrap, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// Exclusive scan of tile counts (one block, up to 32 warps): tile starts,
// the ascending list of non-empty tiles, each tile's slot in it, and the
// first fused-G2P work item of each active tile (ceil(count / kG2PChunk)
// items a tile).  Each warp owns a contiguous chunk of tiles: it sums its
// chunk in coalesced 32-tile steps, one barrier exchanges the warp totals,
// and the warp walks its chunk again with warp-shuffle scans, writing
// coalesced.  (A block-wide scan per 1024 tiles took 32 barrier-bound
// rounds for 32,768 tiles; runs of tiles per thread made every store
// uncoalesced.)
__device__ __forceinline__ int tile_items(int c) { return (c + kG2PChunk - 1) / kG2PChunk; }
__device__ __forceinline__ void tile_scan_block(int ntiles, const int *count, int *start, int *active, int *slot,
                                                int *item_start, Ctl *ctl) {
    constexpr unsigned FULL = 0xffffffffu;
    __shared__ int s_tot[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    const int chunk = ((ntiles + nw - 1) / nw + 31) & ~31;
    const int c0 = min(ntiles, wid * chunk), c1 = min(ntiles, c0 + chunk);
    int tc = 0, ta = 0, ti = 0;
    for (int i = c0 + lane; i < c1; i += 32) {
        const int c = count[i];
        tc += c;
        ta += c > 0;
        ti += tile_items(c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        tc += __shfl_xor_sync(FULL, tc, o);
        ta += __shfl_xor_sync(FULL, ta, o);
        ti += __shfl_xor_sync(FULL, ti, o);
    }
    if (lane == 0) {
        s_tot[0][wid] = tc;
        s_tot[1][wid] = ta;
        s_tot[2][wid] = ti;
    }
    __syncthreads();
    int oc = 0, oa = 0, oi = 0;
    for (int k = 0; k < wid; ++k) {
        oc += s_tot[0][k];
        oa += s_tot[1][k];
        oi += s_tot[2][k];
    }
    for (int base = c0; base < c1; base += 32) {
        const int i = base + lane;
        const int c = i < c1 ? count[i] : 0, a = c > 0, it = tile_items(c);
        int sc = c, sa = a, si = it;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int n1 = __shfl_up_sync(FULL, sc, o), n2 = __shfl_up_sync(FULL, sa, o),
                      n3 = __shfl_up_sync(FULL, si, o);
            if (lane >= o) {
                sc += n1;
                sa += n2;
                si += n3;
            }
        }
        if (i < c1) {
            start[i] = oc + sc - c;
            if (a) {
                const int ai = oa + sa - 1;
                active[ai] = i;
                slot[i] = ai;
                item_start[ai] = oi + si - it;
            } else {
                slot[i] = -1;
            }
        }
        oc += __shfl_sync(FULL, sc, 31);
        oa += __shfl_sync(FULL, sa, 31);
        oi += __shfl_sync(FULL, si, 31);
    }
    if (wid == nw - 1 && lane == 0) {
        // the last warp's offsets now hold the grand totals
        ctl->n_active_tiles = oa;
        ctl->n_sorted = oc;
        ctl->n_g2p_items = oi;
        item_start[oa] = oi;
    }
}
__global__ void k_tile_scan(int ntiles, const int *count, int *start, int *active, int *slot, int *item_start,
                            Ctl *ctl) {
    tile_scan_block(ntiles, count, start, active, slot, item_start, ctl);
}

// Tiles whose owned nodes the nodal kernel writes this step: tiles next to
// a non-empty tile (they receive P2G halo contributions), plus tiles written
// in the previous step (their nodes return to zero, as Reset_Nodaldata_to_Zero
// leaves them).
__device__ __forceinline__ void touched_body(const Params &P, const int *count, int *touched,
                                             long long *touched_step, Ctl *ctl, int t) {
    if (t >= P.ntiles) return;
    int tc[3];
    tile_coords(P, t, tc);
    bool now = false;
    for (int dz = -1; dz <= 1 && !now; ++dz)
        for (int dy = -1; dy <= 1 && !now; ++dy)
            for (int dx = -1; dx <= 1 && !now; ++dx) {
                int s[3] = {tc[0] + dx, tc[1] + dy, tc[2] + dz};
                bool ok = true;
                for (int d = 0; d < 3; ++d) {
                    if (s[d] < 0 || s[d] >= P.ntile[d]) {
                        if (P.periodic[d])
                            s[d] = (s[d] + P.ntile[d]) % P.ntile[d];
                        else
                            ok = false;
                    }
                }
                if (ok && count[(s[2] * P.ntile[1] + s[1]) * P.ntile[0] + s[0]] > 0) now = true;
            }
    long long cur = ctl->steps;
    long long prev = touched_step[t];
    if (now || prev == cur - 1) {
        int idx = atomicAdd(&ctl->n_touched_tiles, 1);
        touched[idx] = t;
    }
    if (now) touched_step[t] = cur;
}
__global__ void k_touched(Params P, const int *count, int *touched, long long *touched_step, Ctl *ctl) {
    touched_body(P, count, touched, touched_step, ctl, blockIdx.x * blockDim.x + threadIdx.x);
}

__device__ __forceinline__ void scatter_body(long long n, const uint32_t *key, int tshift3, const int *start,
                                             int *fill, int32_t *bucket, long long i) {
    int t = -1;
    if (i < n) {
        uint32_t k = key[i];
        if (k != 0xFFFFFFFFu) t = (int)(k >> tshift3);
    }
    unsigned act = __ballot_sync(0xffffffffu, t >= 0);
    const int lane = threadIdx.x & 31;
    const int t0 = __shfl_sync(0xffffffffu, t, 0);
    if (act == 0xffffffffu && __all_sync(0xffffffffu, t == t0)) {
        // the whole warp in one tile (the usual case): one add, lane order
        int base = 0;
        if (lane == 0) base = atomicAdd(&fill[t0], 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        bucket[start[t0] + base + lane] = (int32_t)i;
        return;
    }
    if (t >= 0) {
        unsigned peers = __match_any_sync(act, t);
        int leader = __ffs(peers) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&fill[t], __popc(peers));
        base = __shfl_sync(peers, base, leader);
        int rank = __popc(peers & ((1u << lane) - 1u));
        bucket[start[t] + base + rank] = (int32_t)i;
    }
}
__global__ void k_scatter(long long n, const uint32_t *key, int tshift3, const int *start, int *fill, int32_t *bucket) {
    scatter_body(n, key, tshift3, start, fill, bucket, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// Per-tile stable ordering: particles of one tile sorted by (cell, storage
// index), which equals a stable sort of the whole array by key.
// Entries of a tile sorted in shared memory (larger tiles use the global
// scratch after the bucket array).  5120 (26 KB a block, a tile of 8^3
// bins at ten particles per bin) measured fastest on the dam break, where
// occupancy sets the sort's speed: 0.223 ms against 0.257 ms at 12288 and
// 0.237 / 0.228 / 0.224 ms at 8192 / 6144 / 4608.
constexpr int kSortCap = 5120;
// A cell of up to kRankLinear particles ranks each entry by counting the
// smaller storage indices of its cell (cnt^2 compares, cheapest for the few
// particles of an ordinary cell); a more crowded cell (a pile-up at a wall
// or a contact) is sorted by the whole block instead, in cnt log^2 cnt.
constexpr int kRankLinear = 32;

// Sorts a[0..L) ascending in place with a bitonic network over the next
// power of two P >= L, the whole block taking part.  Each merge first
// compares mirrored positions of a run, then halves, so every comparator
// (i, j) has i < j and puts the smaller value at i; the missing entries
// L..P-1 act as +infinity at the top and therefore never move: a comparator
// with j >= L is skipped.
__device__ void block_bitonic_sort(int32_t *a, int L) {
    int P = 1;
    while (P < L) P <<= 1;
    for (int k = 2; k <= P; k <<= 1) {
        const int hk = k >> 1;
        for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
            const int blk = t / hk, off = t - blk * hk;
            const int i = blk * k + off, j = blk * k + k - 1 - off;
            if (j < L) {
                const int32_t x = a[i], y = a[j];
                if (y < x) {
                    a[i] = y;
                    a[j] = x;
                }
            }
        }
        __syncthreads();
        for (int h = hk >> 1; h >= 1; h >>= 1) {
            for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
                const int blk = t / h, off = t - blk * h;
                const int i = blk * 2 * h + off, j = i + h;
                if (j < L) {
                    const int32_t x = a[i], y = a[j];
                    if (y < x) {
                        a[i] = y;
                        a[j] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// One non-empty tile w of the active list, sorted by the whole block; sm
// holds 3 ncell + kSortCap ints.
__device__ __forceinline__ void tile_sort_item(int *sm, const int *active, const int *start, const int *count,
                                               const uint32_t *key, const int32_t *bucket, int32_t *scratch,
                                               int32_t *perm, int *cell_start, int ncell, Ctl *ctl, int w) {
    int *cnt = sm, *cst = sm + ncell, *fil = sm + 2 * ncell, *ent_s = sm + 3 * ncell;
    __shared__ int sh[34];
    __shared__ int smax;
    const uint32_t cm = (uint32_t)ncell - 1u;
    const int t = active[w];
    const int s0 = start[t], n = count[t];
    int32_t *ent = (n <= kSortCap) ? ent_s : scratch + s0;
    for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
        cnt[c] = 0;
        fil[c] = 0;
    }
    if (threadIdx.x == 0) smax = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) atomicAdd(&cnt[key[bucket[s0 + e]] & cm], 1);
    __syncthreads();
    // exclusive scan of the per-cell counts
    int carry = 0;
    for (int base = 0; base < ncell; base += blockDim.x) {
        int c = base + threadIdx.x;
        int v = c < ncell ? cnt[c] : 0;
        int tot;
        int ex = block_exclusive_scan(v, &tot, sh);
        if (c < ncell) {
            cst[c] = carry + ex;
            if (v > 0) atomicMax(&smax, v);
        }
        carry += tot;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        int i = bucket[s0 + e];
        int c = key[i] & cm;
        ent[cst[c] + atomicAdd(&fil[c], 1)] = i;
    }
    __syncthreads();
    if (smax > kRankLinear) {
        // crowded cells (block-uniform: counts and smax are shared), one
        // after another, each sorted by storage index in place
        for (int c = 0; c < ncell; ++c)
            if (cnt[c] > kRankLinear) block_bitonic_sort(ent + cst[c], cnt[c]);
    }
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        int i = ent[q];
        int c = key[i] & cm;
        int b = cst[c], e = b + cnt[c];
        if (e - b > kRankLinear) {
            perm[s0 + q] = i;  // its cell is sorted already
            continue;
        }
        int rank = 0;
        for (int r = b; r < e; ++r) rank += (ent[r] < i);
        perm[s0 + b + rank] = i;
    }
    // cell ranges of this tile (relative to the tile start), for the
    // per-cell P2G
    int *cs = cell_start + (long long)w * (ncell + 1);
    for (int c = threadIdx.x; c < ncell; c += blockDim.x) cs[c] = cst[c];
    if (threadIdx.x == 0) {
        cs[ncell] = n;
        atomicMax(&ctl->maxppc, smax);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads) k_tile_sort(const int *active, const int *start, const int *count,
                                                        const uint32_t *key, const int32_t *bucket, int32_t *scratch,
                                                        int32_t *perm, int *cell_start, int ncell, Ctl *ctl) {
    extern __shared__ int sm[];
    const int nitems = ctl->n_active_tiles;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x)
        tile_sort_item(sm, active, start, count, key, bucket, scratch, perm, cell_start, ncell, ctl, w);
}

// ---------------------------------------------------------------- bookkeeping
// Start of step: dt from the last particle reduction (Calculate_time_step,
// mpm_particle_timestep.cpp:38-111), current bounds, accumulators reset.
__device__ __forceinline__ void dt_finalize_body(const Params &P, Ctl *ctl, int reset) {
    double dtmin = bitsd(ctl->dtmin_bits);
    double dt;
    if (P.fixed_dt)
        dt = P.timestep;
    else {
        dt = P.cfl * dtmin;
        dt = fmax(fmin(dt, P.dt_max), P.dt_min);
    }
    ctl->dt = dt;
    if (reset) {
        ctl->dtmin_bits = dbits(1.7976931348623157e308);
        for (int c = 0; c < CH_ALL; ++c) ctl->bound_bits[c] = 0ull;
        ctl->lost = 0ull;
        ctl->lost_fill = 0ull;
        ctl->maxppc = 0;
        ctl->n_touched_tiles = 0;
    }
}
__global__ void k_dt_finalize(Params P, Ctl *ctl, int reset) { dt_finalize_body(P, ctl, reset); }

// Fixed-point scales: a channel's node sum is bounded by
// (particles per cell) x (stencil cells) x (largest per-particle term);
// the scale 2^e keeps twice that bound below 2^bits (see fx_add_r).
__device__ __forceinline__ void scales_body(Ctl *ctl, int stencil_cells, int bits, const unsigned long long *bounds,
                                            int c) {
    if (c == 0) ctl->next_p2g = 0;  // the P2G launch that follows takes tiles from 0
    if (c >= CH_ALL) return;
    double b = bitsd(bounds[c]);
    double S = b * (double)(ctl->maxppc > 0 ? ctl->maxppc : 1) * (double)stencil_cells * 2.0;
    double sc = 1.0;
    if (S > 0.0 && S < 1e300) {
        int ex;
        frexp(S, &ex);  // S < 2^ex
        // 2^e stays inside the state's range (FP32: |e| <= 100); a channel
        // this small contributes 0
        const int lim = bits > 64 ? 900 : 100;
        sc = ldexp(1.0, max(-lim, min(lim, bits - ex)));
    }
    ctl->scale[c] = sc;
    ctl->inv_scale[c] = 1.0 / sc;
}
__global__ void k_scales(Ctl *ctl, int stencil_cells, int bits, const unsigned long long *bounds) {
    scales_body(ctl, stencil_cells, bits, bounds, threadIdx.x);
}

__global__ void k_time_advance(Ctl *ctl) {
    ctl->time += ctl->dt;
    ctl->steps += 1;
}

#endif  // EXG_R_FP64

// Reductions over particles that the next step needs before it can start:
// the CFL minimum and the per-channel P2G bounds.
template <class R>
__device__ __forceinline__ void particle_bounds(const Params &P, const Material &mt, double m, const double v[3],
                                                double vol, const double sig[6], double rho, double cp, double T,
                                                double kc, const double q[3], double Q, double b[CH_ALL],
                                                double &speed) {
    b[CH_M] = fabs(m);
    for (int d = 0; d < 3; ++d) b[CH_P + d] = fabs(m * v[d]);
    const int rowi[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (int d = 0; d < 3; ++d) {
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s += fabs(sig[rowi[d][j]]) * 2.0 * P.dxi[j];
        b[CH_F + d] = fabs(m * P.gravity[d]) + (P.external_loads ? fabs(P.extforce[d]) : 0.0) + fabs(vol) * s;
    }
    b[CH_MC] = fabs(m * cp);
    b[CH_MCT] = fabs(m * cp * T);
    b[CH_MK] = fabs(m * kc);
    double sq = 0.0;
    for (int d = 0; d < 3; ++d) sq += fabs(q[d]) * 2.0 * P.dxi[d];
    b[CH_SRC] = fabs(vol) * sq + fabs(vol * Q);
    // Calculate_time_step, mpm_particle_timestep.cpp:55-100 (the modulus per
    // material, Material::pmod)
    const double Cs = sqrt(mt.pmod / rho);
    double vm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    // the particle's CFL step is dxmin / speed; a thread that handles many
    // particles keeps the largest speed and divides once: correctly rounded
    // division by a positive number is monotone, so the minimum step is the
    // same bits
    speed = Cs + vm;
}

// The same reductions in the mixed-precision G2P without temperature, in
// FP32: the bounds only set power-of-two fixed-point scales with a factor-2
// margin, so FP32 rounded upward bounds them as well; the CFL speed is the
// FP32 sum of FP32 square roots (dt then carries a relative 1e-7 of FP32
// rounding, as the FP32 velocities it follows).  Saves the FP64 divisions,
// square roots and channel sums of particle_bounds.
__device__ __forceinline__ void lean_bounds_f(const Params &P, const Material &mt, float m, const float v[3],
                                              float vol, const float sig[6], float rho, float (&run_b)[CH_ALL],
                                              double &run_speed) {
    const float am = fabsf(m), av = fabsf(vol);
    run_b[CH_M] = fmaxf(run_b[CH_M], am);
#pragma unroll
    for (int d = 0; d < 3; ++d) run_b[CH_P + d] = fmaxf(run_b[CH_P + d], __fmul_ru(am, fabsf(v[d])));
    const int rowi[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float s = 0.f;
#pragma unroll
        for (int j = 0; j < 3; ++j) s = __fadd_ru(s, __fmul_ru(fabsf(sig[rowi[d][j]]), __double2float_ru(2.0 * P.dxi[j])));
        float b = __fmul_ru(am, __double2float_ru(fabs(P.gravity[d])));
        if (P.external_loads) b = __fadd_ru(b, __double2float_ru(fabs(P.extforce[d])));
        b = __fadd_ru(b, __fmul_ru(av, s));
        run_b[CH_F + d] = fmaxf(run_b[CH_F + d], b);
    }
    const float cs = sqrtf(__double2float_rn(mt.pmod) / rho);
    const float vm = sqrtf(fmaf(v[2], v[2], fmaf(v[1], v[1], v[0] * v[0])));
    run_speed = fmax(run_speed, (double)(cs + vm));
}

__device__ __forceinline__ void block_reduce_push(unsigned long long *bounds, unsigned long long *dtmin,
                                                  double b[CH_ALL], double dtp, bool valid) {
    __shared__ unsigned long long red[CH_ALL + 1][32];  // any block of up to 1024 threads
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c = 0; c < CH_ALL; ++c) {
        unsigned long long u = valid ? dbits(b[c]) : 0ull;
        u = warp_max_u64(u);
        if (lane == 0) red[c][wid] = u;
    }
    unsigned long long ud = valid ? dbits(dtp) : dbits(1.7976931348623157e308);
    ud = warp_min_u64(ud);
    if (lane == 0) red[CH_ALL][wid] = ud;
    __syncthreads();
    if (threadIdx.x < CH_ALL) {
        unsigned long long m = 0ull;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = red[threadIdx.x][w] > m ? red[threadIdx.x][w] : m;
        if (m) atomicMax(&bounds[threadIdx.x], m);
    } else if (threadIdx.x == CH_ALL) {
        unsigned long long m = ~0ull;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = red[CH_ALL][w] < m ? red[CH_ALL][w] : m;
        atomicMin(dtmin, m);
    }
}

template <class R>
__global__ void __launch_bounds__(kThreads) k_state_reduce(Params P, Parts<R> A, const Material *mats, long long n,
                                                           unsigned long long *bounds, unsigned long long *dtmin) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool valid = false;
    double b[CH_ALL] = {};
    double dtp = 0.0;
    if (p < n && A.phase[p] == 0) {
        double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
        int iv[3];
        cell_of(P, x, iv);
        valid = true;
        for (int d = 0; d < 3; ++d) valid = valid && iv[d] >= 0 && iv[d] < P.nc[d];
        if (valid) {
            double v[3] = {(double)A.v[0][p], (double)A.v[1][p], (double)A.v[2][p]};
            double s[6];
            for (int c = 0; c < 6; ++c) s[c] = (double)A.sig[c][p];
            double q[3] = {0, 0, 0}, cp = 0, T = 0, kc = 0, Q = 0;
            if (P.use_temp) {
                for (int d = 0; d < 3; ++d) q[d] = (double)A.q[d][p];
                cp = A.cp[p];
                T = A.T[p];
                kc = A.kc[p];
                Q = A.Q[p];
            }
            double speed;
            particle_bounds<R>(P, mats[A.mat[p]], (double)A.mass[p], v, (double)A.vol[p], s, (double)A.rho[p], cp, T,
                               kc, q, Q, b, speed);
            dtp = P.dxmin / speed;
        }
    }
    block_reduce_push(bounds, dtmin, b, dtp, valid);
}

#if defined(EXG_R_FP64)
__global__ void k_reset_accum(unsigned long long *bounds, unsigned long long *dtmin) {
    if (threadIdx.x < CH_ALL) bounds[threadIdx.x] = 0ull;
    if (threadIdx.x == 0) *dtmin = dbits(1.7976931348623157e308);
}
#endif

// ---------------------------------------------------------------- K2 P2G
// deposit_onto_grid_momentum (mpm_particle_grid_ops.cpp:405-588) and the
// thermal deposit (:703-844), one CTA per non-empty tile.  Contributions are
// converted to 64-bit fixed point with a per-channel power-of-two scale and
// accumulated with integer shared-memory atomics: integer addition is
// associative, so node sums do not depend on thread scheduling and the
// result is identical run to run.  The CTA then stores its whole node block
// (tile plus halo) as one partial; the nodal kernel adds the <= 8 partials
// covering each node.
template <int ORD>
struct Stc {
    static constexpr int W = (ORD == 1) ? 2 : 4;
    static constexpr int LO = (ORD == 1) ? 0 : -1;
};

template <int W, class T>
__device__ __forceinline__ T pick(const T (&a)[W], int i) {
    if (W == 2) return i ? a[1] : a[0];
    return i == 0 ? a[0] : (i == 1 ? a[1] : (i == 2 ? a[2] : a[W - 1]));
}

// ---------------------------------------------------------------- K2 per-cell P2G
// P2G with one thread per cell (nearest-node bin for quadratic): the thread
// walks its cell's particles (contiguous after the sort) in storage order
// and accumulates their contributions to rows of one z-slice of the cell's
// stencil in registers; only the per-cell sums go to the tile's node block
// in shared memory, as 64-bit fixed point.  The summation order inside a
// cell is fixed and the cross-cell sums are exact, so the result is
// deterministic; shared-memory atomics drop by the particles-per-cell factor
// and lanes never collide (a warp's lanes own different cells and add the
// same stencil offset at the same time).
template <class R>
__device__ __forceinline__ long long to_fixed(R v, R sc);
template <>
__device__ __forceinline__ long long to_fixed<float>(float v, float sc) {
    return __float2ll_rn(v * sc);
}
template <>
__device__ __forceinline__ long long to_fixed<double>(double v, double sc) {
    return __double2ll_rn(v * sc);
}

// A node's fixed-point sum in shared memory.
// FP32 state (scale bound 2^55, kFxBits32): two 32-bit words; without
// carries, lo collects the low 24 bits of each addend (at most 64 addends
// per node and tile, so lo < 2^30) and hi the arithmetic upper part, which
// fits 32 bits; the value is hi * 2^24 + lo and both adds are
// fire-and-forget reductions.
// FP64 state (bound 2^93, kFxBits64): a 64-bit low word and a 32-bit high
// word, value hi * 2^64 + lo; the low word's returning add yields the carry.
// The 93 bits keep the FP64 mantissa of a node whose sum is 2^-40 of the
// channel's bound: a node reached only by the edge of a few particles'
// supports has a mass that small, and its velocity p / m, which the
// velocity gradient weights by the slowly vanishing dN, needs relative, not
// absolute, precision.
constexpr int kFxBits32 = 55, kFxBits64 = 93;
// 32-bit words of the low part of one fixed-point value (shared memory)
template <class R>
__host__ __device__ constexpr int fx_lo_words() { return sizeof(R) == 4 ? 1 : 2; }

// The FP64 addend x = v * sc (|x| < 2^93) as hi * 2^64 + lo.  Below 2^63 in
// magnitude it is the rounded 64-bit integer, sign-extended; above, x is an
// integer already and hi = floor(x / 2^64) and lo = x - hi 2^64 are exact.
// Both are formed and one is selected (no divergence).
__device__ __forceinline__ void fx_split64(double x, unsigned long long &lo, int &hi) {
    const long long q = __double2ll_rn(x);
    const double h = floor(x * 0x1p-64);
    const double r = fma(-h, 0x1p64, x);
    const bool small = fabs(x) < 0x1p63;
    lo = small ? (unsigned long long)q : __double2ull_rn(r);
    hi = small ? (q < 0 ? -1 : 0) : (int)h;
}

// Branch-free: adding zero words changes no sum, and the straight-line
// code keeps a warp's lanes together.
template <class R>
__device__ __forceinline__ void fx_add_r(unsigned *lo, int *hi, int idx, R v, R sc) {
    if (sizeof(R) == 4) {
        const long long q = to_fixed<R>(v, sc);
        atomicAdd(&lo[idx], (unsigned)(q & 0xFFFFFFll));
        atomicAdd(&hi[idx], (int)(q >> 24));
    } else {
        unsigned long long l;
        int h;
        fx_split64((double)v * (double)sc, l, h);
        unsigned long long *lo64 = reinterpret_cast<unsigned long long *>(lo);
        const unsigned long long old = atomicAdd(&lo64[idx], l);
        atomicAdd(&hi[idx], h + ((old + l < old) ? 1 : 0));
    }
}
// Zeroes the tile's fixed-point block (n values) in shared memory.
template <class R>
__device__ __forceinline__ void fx_zero(unsigned *lo, int *hi, int n) {
    for (int i = threadIdx.x; i < n * fx_lo_words<R>(); i += blockDim.x) lo[i] = 0u;
    for (int i = threadIdx.x; i < n; i += blockDim.x) hi[i] = 0;
}
// Writes the tile's fixed-point block (n values) to its staging slot: FP32
// one 64-bit integer per value; FP64 the 64-bit low words, then the 32-bit
// high words.
template <class R>
__device__ __forceinline__ void fx_store(const unsigned *lo, const int *hi, int n, long long *dst) {
    if (sizeof(R) == 4) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = (long long)hi[i] * (1ll << 24) + (long long)lo[i];
    } else {
        const unsigned long long *lo64 = reinterpret_cast<const unsigned long long *>(lo);
        int *dh = reinterpret_cast<int *>(dst + n);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            dst[i] = (long long)lo64[i];
            dh[i] = hi[i];
        }
    }
}
// A node's sum over its partial blocks: FP32 a 64-bit integer; FP64 a 128-bit
// two's-complement pair (hi carries the low words' overflow).
template <class R>
struct FxSum {
    long long v = 0;
    __device__ __forceinline__ void add(const long long *blk, long long nv, long long i) { v += blk[i]; }
    __device__ __forceinline__ double value() const { return (double)v; }
};
template <>
struct FxSum<double> {
    unsigned long long lo = 0;
    long long hi = 0;
    __device__ __forceinline__ void add(const long long *blk, long long nv, long long i) {
        const unsigned long long l = (unsigned long long)blk[i];
        const int h = reinterpret_cast<const int *>(blk + nv)[i];
        const unsigned long long o = lo;
        lo = o + l;
        hi += (long long)h + (lo < o ? 1 : 0);
    }
    // exact below 2^63 in magnitude; above, (double)lo rounds by at most 2^10
    // against a value of at least 2^63, then the sum rounds once
    __device__ __forceinline__ double value() const {
        if ((hi == 0 && (long long)lo >= 0) || (hi == -1 && (long long)lo < 0)) return (double)(long long)lo;
        return (double)hi * 0x1p64 + (double)lo;
    }
};

// Stencil width of the per-cell P2G: cells (linear, cubic, mixed orders) or
// nearest-node bins (uniform quadratic).  The block index of stencil slot s
// is (local cell or bin) + s in every case.
template <int ORD>
struct P2GStc {
    static constexpr int W = (ORD == 1) ? 2 : (ORD == 2 ? 3 : 4);
};

// FP32 state: the interior B-spline pieces in forms without cancellation.
// The reference evaluates the expanded pieces (a z^2 + b z + c, and the
// cubic's a z^3 + ...) in FP64, whose rounding where a piece falls to zero
// at the support's edge is ~1e-16 absolute.  In FP32 the same expansion
// leaves ~1e-7 absolute there, against a true weight of (1/2) t^2 = 5e-9
// for a particle t = 1e-4 inside a quadratic support's edge: the node's
// weight, and with it its mass, comes out negative or many times too large,
// its velocity p / m is garbage, and the next steps blow up (particles
// started on a lattice sit exactly on such edges).  Factored, every weight
// keeps FP32's relative precision: quadratic (1/2)(1/2 - u)^2, 3/4 - u^2,
// (1/2)(1/2 + u)^2; cubic g^3 / 6, 2/3 + f^2 (f / 2 - 1),
// 2/3 + g^2 (g / 2 - 1), f^3 / 6 with g = 1 - f.  The reference's truncated
// constants round to the same floats as 1/6 and 2/3.  Per slot s (unscaled
// derivative):
__device__ __forceinline__ void slot_weight_f32(int ord, float f, int s, float &w, float &dw) {
    if (ord == 3) {
        const float t = (s == 0 || s == 2) ? 1.f - f : f, t2 = t * t;
        if (s == 0 || s == 3) {
            w = t2 * (t * (float)kOneBySix);
            dw = (s == 0 ? -0.5f : 0.5f) * t2;
        } else {
            w = fmaf(t2, fmaf(0.5f, t, -1.f), (float)kTwoByThree);
            dw = (s == 1 ? t : -t) * fmaf(1.5f, t, -2.f);
        }
    } else if (s == 1) {
        w = fmaf(-f, f, 0.75f);
        dw = -2.f * f;
    } else {
        const float t = s == 0 ? 0.5f - f : 0.5f + f;
        w = 0.5f * (t * t);
        dw = s == 0 ? -t : t;
    }
}

// Interior weights of all W slots from the particle's offset f in its cell
// (cubic, slot s at z = f + 1 - s) or bin (quadratic, u = offset from the
// bin's node, slot s at u + 1 - s): the fixed pieces of the type-3 splines,
// the same coefficients as the tables (FP64), or their factored forms (FP32,
// two slots per packed instruction).
template <class R, int ORD>
__device__ __forceinline__ void interior_weights(R f, R dxinv, AxisW<R, P2GStc<ORD>::W> &a) {
    if constexpr (ORD == 3 && sizeof(R) == 4) {
        const float o6 = (float)kOneBySix, t3 = (float)kTwoByThree, g = 1.f - f;
        // end slots (0, 3) in t = (g, f), middle slots (1, 2) in t = (f, g)
        const float2 e = make_float2(g, f), c = make_float2(f, g);
        const float2 e2 = __fmul2_rn(e, e), c2 = __fmul2_rn(c, c);
        const float2 we = __fmul2_rn(e2, __fmul2_rn(e, make_float2(o6, o6)));
        const float2 wc = __ffma2_rn(c2, __ffma2_rn(make_float2(0.5f, 0.5f), c, make_float2(-1.f, -1.f)),
                                     make_float2(t3, t3));
        const float2 de = __fmul2_rn(e2, make_float2(-0.5f * dxinv, 0.5f * dxinv));
        const float2 dc = __fmul2_rn(__fmul2_rn(c, __ffma2_rn(make_float2(1.5f, 1.5f), c, make_float2(-2.f, -2.f))),
                                     make_float2(dxinv, -dxinv));
        a.w[0] = we.x;
        a.w[1] = wc.x;
        a.w[2] = wc.y;
        a.w[3] = we.y;
        a.dw[0] = de.x;
        a.dw[1] = dc.x;
        a.dw[2] = dc.y;
        a.dw[3] = de.y;
    } else if constexpr (ORD == 2 && sizeof(R) == 4) {
        const float2 t = make_float2(0.5f - f, 0.5f + f);
        const float2 wt = __fmul2_rn(make_float2(0.5f, 0.5f), __fmul2_rn(t, t));
        a.w[0] = wt.x;
        a.w[1] = fmaf(-f, f, 0.75f);
        a.w[2] = wt.y;
        a.dw[0] = -t.x * dxinv;
        a.dw[1] = (-2.f * f) * dxinv;
        a.dw[2] = t.y * dxinv;
    } else if constexpr (ORD == 3) {
        const R o6 = (R)kOneBySix, t3 = (R)kTwoByThree, f3 = (R)kFourByThree;
        R z = f + R(1), z2 = z * z;
        a.w[0] = fma(-o6, z2 * z, fma(R(1), z2, fma(R(-2), z, f3)));
        a.dw[0] = fma(R(-0.5), z2, fma(R(2), z, R(-2))) * dxinv;
        z = f;
        z2 = z * z;
        a.w[1] = fma(R(0.5), z2 * z, fma(R(-1), z2, fma(R(0), z, t3)));
        a.dw[1] = fma(R(1.5), z2, fma(R(-2), z, R(0))) * dxinv;
        z = f - R(1);
        z2 = z * z;
        a.w[2] = fma(R(-0.5), z2 * z, fma(R(-1), z2, fma(R(0), z, t3)));
        a.dw[2] = fma(R(-1.5), z2, fma(R(-2), z, R(0))) * dxinv;
        z = f - R(2);
        z2 = z * z;
        a.w[3] = fma(o6, z2 * z, fma(R(1), z2, fma(R(2), z, f3)));
        a.dw[3] = fma(R(0.5), z2, fma(R(2), z, R(2))) * dxinv;
    } else {
        // quadratic on the bin's nodes n0 - 1, n0, n0 + 1 (pieces
        // [0.5, 1.5], [-0.5, 0.5], [-1.5, -0.5])
        R z = f + R(1);
        a.w[0] = fma(R(0.5), z * z, fma(R(-1.5), z, R(1.125)));
        a.dw[0] = (z - R(1.5)) * dxinv;
        z = f;
        a.w[1] = fma(R(-1), z * z, fma(R(0), z, R(0.75)));
        a.dw[1] = (R(-2) * z) * dxinv;
        z = f - R(1);
        a.w[2] = fma(R(0.5), z * z, fma(R(1.5), z, R(1.125)));
        a.dw[2] = (z + R(1.5)) * dxinv;
    }
}

// Per-axis weights of a cell whose stencil nodes are all interior (shape
// type 3): the polynomial piece of each stencil offset is fixed (linear,
// cubic; quadratic uses dual_axis_weights); same coefficients as the tables.
template <class R, int ORD>
__device__ __forceinline__ void axis_weights_interior(const Params &P, int d, double x, int i,
                                                      AxisW<R, Stc<ORD>::W> &a) {
    const double fd = (x - (P.plo[d] + i * P.dx[d])) * P.dxi[d];
    const R f = (R)fd;
    const R dxinv = (R)P.dxi[d];
    if (ORD == 1) {
        a.w[0] = (R)(1.0 - fd);  // formed in FP64: relative precision as the weight vanishes
        a.w[1] = f;
        a.dw[0] = -dxinv;
        a.dw[1] = dxinv;
    } else if constexpr (sizeof(R) == 4 && ORD == 3) {
        interior_weights<R, 3>(f, dxinv, a);  // factored pieces (FP32)
    } else {
        // type-3 cubic pieces, interval 3 - s for stencil slot s
        const R o6 = (R)kOneBySix, t3 = (R)kTwoByThree, f3 = (R)kFourByThree;
        R z = f + R(1), z2 = z * z;
        a.w[0] = -o6 * (z2 * z) + R(1) * z2 + R(-2) * z + f3;
        a.dw[0] = (R(-0.5) * z2 + R(2) * z + R(-2)) * dxinv;
        z = f;
        z2 = z * z;
        a.w[1] = R(0.5) * (z2 * z) + R(-1) * z2 + R(0) * z + t3;
        a.dw[1] = (R(1.5) * z2 + R(-2) * z + R(0)) * dxinv;
        z = f - R(1);
        z2 = z * z;
        a.w[2] = R(-0.5) * (z2 * z) + R(-1) * z2 + R(0) * z + t3;
        a.dw[2] = (R(-1.5) * z2 + R(-2) * z + R(0)) * dxinv;
        z = f - R(2);
        z2 = z * z;
        a.w[3] = o6 * (z2 * z) + R(1) * z2 + R(2) * z + f3;
        a.dw[3] = (R(0.5) * z2 + R(2) * z + R(2)) * dxinv;
    }
}

template <class R, int ORD>
__device__ __forceinline__ void cell_axis_weights(const SplineTables &tab, const Params &P, int d, double x, int i,
                                                  bool interior, AxisW<R, Stc<ORD>::W> &a) {
    if (ORD != 0 && interior)
        axis_weights_interior<R, ORD>(P, d, x, i, a);
    else
        axis_weights<R, Stc<ORD>::W, Stc<ORD>::LO>(tab, P, d, x, i, a);
}

// Quadratic weights on the 3-node window bin-1..bin+1 of a nearest-node bin
// (dual_bin).  Interior bins (all three nodes of shape type 3) use the fixed
// pieces; elsewhere each node's own piece comes from the tables, and nodes
// outside the domain get 0, which is what compute_bounds leaves out
// (mpm_particle_grid_ops.cpp:255-299): every in-domain node outside the
// window is at least 1.5 dx away and has weight 0 for every shape type.
template <class R>
__device__ __forceinline__ void dual_axis_weights(const SplineTables &tab, const Params &P, int d, double x, int n0,
                                                  bool interior, AxisW<R, 3> &a) {
    const R dxinv = (R)P.dxi[d];
    if (interior) {
        const R u = (R)((x - (P.plo[d] + n0 * P.dx[d])) * P.dxi[d]);
        if constexpr (sizeof(R) == 4) {
            interior_weights<R, 2>(u, dxinv, a);  // factored pieces (FP32)
            return;
        }
        R z = u + R(1);  // node n0-1, piece [0.5, 1.5]
        a.w[0] = R(0.5) * z * z + R(-1.5) * z + R(1.125);
        a.dw[0] = (z - R(1.5)) * dxinv;
        z = u;  // node n0, piece [-0.5, 0.5]
        a.w[1] = R(-1) * z * z + R(0) * z + R(0.75);
        a.dw[1] = (R(-2) * z) * dxinv;
        z = u - R(1);  // node n0+1, piece [-1.5, -0.5]
        a.w[2] = R(0.5) * z * z + R(1.5) * z + R(1.125);
        a.dw[2] = (z + R(1.5)) * dxinv;
        return;
    }
#pragma unroll
    for (int s = 0; s < 3; ++s) {
        const int n = n0 - 1 + s;
        R val = R(0), der = R(0);
        if (P.periodic[d] || (n >= 0 && n <= P.nc[d])) {
            const int ty = shape_type(n, P.nc[d], P.periodic[d]);
            const double r = (x - (P.plo[d] + n * P.dx[d])) * P.dxi[d];
            spline_eval<R>(tab, 2, ty, r, val, der);
            der *= dxinv;
        }
        a.w[s] = val;
        a.dw[s] = der;
    }
}

template <class R, int ORD>
__device__ __forceinline__ void p2g_axis_weights(const SplineTables &tab, const Params &P, int d, double x, int i,
                                                 bool interior, AxisW<R, P2GStc<ORD>::W> &a) {
    if constexpr (ORD == 2)
        dual_axis_weights<R>(tab, P, d, x, i, interior, a);
    else
        cell_axis_weights<R, ORD>(tab, P, d, x, i, interior, a);
}

// Per-particle P2G coefficients: m, m v, the body force m g (+ the external
// force inside the slab) and -V sigma, so that every node contribution is a
// chain of fused multiply-adds; thermal: m cp, m cp T, m k, V q, V Q.
template <class R, bool THERM>
struct P2GCoef {
    R m, mv[3], b[3], s[6];
    R mcp, mcpT, mk, qv[3], VQ;
};

// Register accumulators of one stencil node.  FP32 keeps channel pairs in
// float2 and adds them with the packed FP32 FMA of sm_100 (two lanes per
// instruction): (m, p_x), (p_y, p_z), (f_x, f_y), then f_z alone.
template <class R, bool THERM>
struct P2GAcc {
    R c[THERM ? CH_ALL : CH_MOM_END];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < (THERM ? CH_ALL : CH_MOM_END); ++i) c[i] = R(0);
    }
    __device__ __forceinline__ void add(const P2GCoef<R, THERM> &q, R N, R g0, R g1, R g2) {
        c[CH_M] = fma(q.m, N, c[CH_M]);
#pragma unroll
        for (int d = 0; d < 3; ++d) c[CH_P + d] = fma(q.mv[d], N, c[CH_P + d]);
        c[CH_F + 0] = fma(q.s[2], g2, fma(q.s[1], g1, fma(q.s[0], g0, fma(q.b[0], N, c[CH_F + 0]))));
        c[CH_F + 1] = fma(q.s[4], g2, fma(q.s[3], g1, fma(q.s[1], g0, fma(q.b[1], N, c[CH_F + 1]))));
        c[CH_F + 2] = fma(q.s[5], g2, fma(q.s[4], g1, fma(q.s[2], g0, fma(q.b[2], N, c[CH_F + 2]))));
        if (THERM) add_thermal(q, N, g0, g1, g2);
    }
    __device__ __forceinline__ void add_thermal(const P2GCoef<R, THERM> &q, R N, R g0, R g1, R g2) {
        if constexpr (THERM) {
            c[CH_MC] = fma(q.mcp, N, c[CH_MC]);
            c[CH_MCT] = fma(q.mcpT, N, c[CH_MCT]);
            c[CH_MK] = fma(q.mk, N, c[CH_MK]);
            c[CH_SRC] = fma(q.VQ, N, fma(q.qv[2], g2, fma(q.qv[1], g1, fma(q.qv[0], g0, c[CH_SRC]))));
        }
    }
    __device__ __forceinline__ R get(int ch) const { return c[ch]; }
};

template <bool THERM>
struct P2GAcc<float, THERM> {
    float2 mp0, p12, f01;
    float f2;
    float th[4];  // m cp, m cp T, m k, source
    __device__ __forceinline__ void zero() {
        mp0 = p12 = f01 = make_float2(0.f, 0.f);
        f2 = 0.f;
#pragma unroll
        for (int i = 0; i < 4; ++i) th[i] = 0.f;
    }
    // N, g0, g1, g2 arrive as broadcast pairs (both lanes equal)
    __device__ __forceinline__ void add2(const float2 cm, const float2 cp, const float2 cb, const float2 cs0,
                                         const float2 cs1, const float2 cs2, const P2GCoef<float, THERM> &q,
                                         float2 NN, float2 G0, float2 G1, float2 G2) {
        mp0 = __ffma2_rn(cm, NN, mp0);
        p12 = __ffma2_rn(cp, NN, p12);
        f01 = __ffma2_rn(cb, NN, f01);
        f01 = __ffma2_rn(cs0, G0, f01);
        f01 = __ffma2_rn(cs1, G1, f01);
        f01 = __ffma2_rn(cs2, G2, f01);
        f2 = fmaf(q.s[5], G2.x, fmaf(q.s[4], G1.x, fmaf(q.s[2], G0.x, fmaf(q.b[2], NN.x, f2))));
        if constexpr (THERM) {
            th[0] = fmaf(q.mcp, NN.x, th[0]);
            th[1] = fmaf(q.mcpT, NN.x, th[1]);
            th[2] = fmaf(q.mk, NN.x, th[2]);
            th[3] = fmaf(q.VQ, NN.x, fmaf(q.qv[2], G2.x, fmaf(q.qv[1], G1.x, fmaf(q.qv[0], G0.x, th[3]))));
        }
    }
    __device__ __forceinline__ float get(int ch) const {
        switch (ch) {
            case CH_M: return mp0.x;
            case CH_P: return mp0.y;
            case CH_P + 1: return p12.x;
            case CH_P + 2: return p12.y;
            case CH_F: return f01.x;
            case CH_F + 1: return f01.y;
            case CH_F + 2: return f2;
            default: return th[ch - CH_MC];
        }
    }
};

constexpr int kCellThreads = 128;
// launch shapes of the quadratic P2G and of the fused G2P (threads per
// block, minimum resident blocks per SM for the register cap); the fused
// G2P measured fastest at 2 x 256 (128 registers) against 1 x 256, 4 x 128,
// 3 x 128, 3 x 256, 2 x 384 and 1 x 512
constexpr int kMaxTileCells = 512;  // T^3 for the largest tile side, 8
#ifndef EXG_P2G2_THREADS
#define EXG_P2G2_THREADS 512
#endif
#ifndef EXG_P2G2_MINB
#define EXG_P2G2_MINB 1
#endif
#ifndef EXG_G2P_THREADS
#define EXG_G2P_THREADS 256
#endif
// Quadratic momentum P2G with the z-slices split across threads, a bin's
// three slices in adjacent threads (FP32 P2G 0.77 ms on the dam break
// against 1.01 ms unsplit and 0.87 ms with the slices in separate thirds of
// the block; FP64 1.47 against 2.51 ms unsplit)
#ifndef EXG_P2G_SPLIT
#define EXG_P2G_SPLIT 1
#endif
// L2 prefetch, at the start of each bin, of the first particle of the bin
// the thread takes next (P2G 0.87-0.90 ms against 0.91 ms without)
#ifndef EXG_P2G_PREFETCH
#define EXG_P2G_PREFETCH 1
#endif

#ifndef EXG_G2P_MINB
#define EXG_G2P_MINB 2
#endif

// Threads per block and register cap of the per-cell P2G: the 3-wide
// quadratic accumulators fit 128 registers; one 512-thread block per SM (a
// thread per bin of an 8^3 tile) measured fastest on the dam break, ahead
// of 2 x 256, 4 x 128 and 1 x 256 with 255 registers.
// Launch variants of the factorized momentum P2G (uniform quadratic and
// cubic): rows per pass, threads per block and the minimum resident blocks
// per SM (the register cap).  Variant 0 is the default; the autotuner
// measures all kP2GVariants on the context's own particles and keeps the
// fastest.  FP32 cubic holds a 4 x 4 slice (112 accumulators, one 256-thread
// block per SM; half slices at 16 warps per SM measured 35 % slower); FP64
// holds one or two rows.
constexpr int kP2GVariants = 3;
static_assert(kP2GVariants == EXG_NUM_VARIANTS, "the launchers dispatch EXG_NUM_VARIANTS P2G variants");
// rows per pass, threads per block, minimum blocks per SM, lane map (0: a
// warp takes one z-slice of 32 cells, 1: a cell's slices in adjacent
// lanes), channel groups (2: mass and momentum apart from force)
//   FP32 cubic:     (4, 256, 1, 0, 1)  (4, 256, 1, 1, 1)  (4, 256, 2, 0, 2)
//   FP32 quadratic: (3, 512, 1, 0, 1)  (3, 512, 1, 1, 1)  (3, 256, 2, 0, 1)
//   FP64 cubic:     (1, 512, 1, 1, 1)  (2, 256, 1, 1, 1)  (1, 512, 1, 0, 1)
//   FP64 quadratic: (1, 512, 1, 1, 1)  (3, 256, 1, 1, 1)  (1, 512, 1, 0, 1)
template <class R, int ORD, int V>
struct P2GVar {
    static constexpr int K = (sizeof(R) == 4 ? 0 : 2) + (ORD == 3 ? 0 : 1);
    static constexpr int TAB[4][3][5] = {{{4, 256, 1, 0, 1}, {4, 256, 1, 1, 1}, {4, 256, 2, 0, 2}},
                                         {{3, 512, 1, 0, 1}, {3, 512, 1, 1, 1}, {3, 256, 2, 0, 1}},
                                         {{1, 512, 1, 1, 1}, {2, 256, 1, 1, 1}, {1, 512, 1, 0, 1}},
                                         {{1, 512, 1, 1, 1}, {3, 256, 1, 1, 1}, {1, 512, 1, 0, 1}}};
    static constexpr int ROWS = TAB[K][V][0], THREADS = TAB[K][V][1], MINB = TAB[K][V][2], MAP = TAB[K][V][3];
    static constexpr int GROUPS = TAB[K][V][4];
};

template <class R, int ORD, bool THERM>
struct P2GCfg {
    static constexpr int W = P2GStc<ORD>::W;
    static constexpr bool FACT = (ORD == 2 || ORD == 3) && !THERM;
    // y rows of the stencil slice accumulated per pass (register budget)
    static constexpr int ROWS = FACT ? P2GVar<R, (FACT ? ORD : 2), 0>::ROWS
                                     : ((sizeof(R) == 8) ? 1 : (THERM ? (W == 4 ? 2 : 1) : W));
    // quadratic momentum: the three z-slices of a bin's window go to three
    // adjacent threads (FP32: one pass each, FP64: one pass per y row)
    // instead of one thread walking them in turn, so the bin's particles are
    // read by the three together and stay in L1
    static constexpr bool SPLIT = EXG_P2G_SPLIT && ORD == 2 && !THERM;
    static constexpr int THREADS = FACT ? P2GVar<R, (FACT ? ORD : 2), 0>::THREADS
                                        : ((ORD == 2) ? EXG_P2G2_THREADS : kCellThreads);
    static constexpr int MINB = FACT ? P2GVar<R, (FACT ? ORD : 2), 0>::MINB : ((ORD == 2) ? EXG_P2G2_MINB : 1);
    static constexpr int MAP = FACT ? P2GVar<R, (FACT ? ORD : 2), 0>::MAP : 0;
};

// One tile of the per-cell P2G into its fixed-point node block (zeroed by
// the caller) and from there to the tile's staging slot.
template <class R, int ORD, bool THERM>
__device__ __forceinline__ void p2g_tile(const SplineTables *tab, unsigned *acc_lo, int *acc_hi, const Params &P,
                                         const Parts<R> &A, const int *active, const int *start, const int *cell_start,
                                         const int32_t *perm, long long *staging, const R *sc, const R *grav, int w) {
    constexpr int W = P2GCfg<R, ORD, THERM>::W;
    constexpr int NCH = THERM ? CH_ALL : CH_MOM_END;
    constexpr int ROWS = P2GCfg<R, ORD, THERM>::ROWS;
    const int B = P.B, B3 = B * B * B, T = P.T, T3 = T * T * T;
    const int t = active[w];
    int tc[3];
    tile_coords(P, t, tc);
    const int s0 = start[t];
    const int *cs = cell_start + (long long)w * (T3 + 1);
    constexpr bool SPLIT = P2GCfg<R, ORD, THERM>::SPLIT;
    // split: tasks (bin, slice) with the three slices of a bin in adjacent
    // threads, so they read the bin's particles together and every thread of
    // a 512-thread block takes exactly three tasks of an 8^3 tile
    const int ntask = SPLIT ? W * T3 : T3, step = (int)blockDim.x;
    for (int u = threadIdx.x; u < ntask; u += step) {
        const int c = SPLIT ? u / W : u;
        const int sz_lo = SPLIT ? u - c * W : 0, sz_hi = SPLIT ? sz_lo + 1 : W;
        const int cnext = SPLIT ? (u + step) / W : u + step;
        const int ka = cs[c], kb = cs[c + 1];
        if (EXG_P2G_PREFETCH && sz_lo == 0 && cnext < T3) {
            // L2 prefetch of the first particle of the bin this thread takes next
            const int kn = cs[cnext];
            if (kn < cs[cnext + 1]) {
                const int pn = perm[s0 + kn];
                auto pf = [](const void *q) { asm volatile("prefetch.global.L2 [%0];" ::"l"(q)); };
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    pf(A.x[d] + pn);
                    pf(A.v[d] + pn);
                }
#pragma unroll
                for (int c6 = 0; c6 < 6; ++c6) pf(A.sig[c6] + pn);
                pf(A.mass + pn);
                pf(A.vol + pn);
                pf(A.phase + pn);
            }
        }
        if (ka == kb) continue;
        const int lx = c % T, ly = (c / T) % T, lz = c / (T * T);
        const int iv[3] = {tc[0] * T + lx, tc[1] * T + ly, tc[2] * T + lz};
        bool inter[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            inter[d] = (ORD == 1) || P.periodic[d] ||
                       (ORD == 2 ? (iv[d] >= 3 && iv[d] <= P.nc[d] - 3) : (iv[d] >= 3 && iv[d] <= P.nc[d] - 4));
        for (int sz = sz_lo; sz < sz_hi; ++sz) {
#pragma unroll
            for (int sy0 = 0; sy0 < W; sy0 += ROWS) {
                P2GAcc<R, THERM> acc[ROWS][W];
#pragma unroll
                for (int r = 0; r < ROWS; ++r)
#pragma unroll
                    for (int sx = 0; sx < W; ++sx) acc[r][sx].zero();
                bool any = false;
                for (int k = ka; k < kb; ++k) {
                    const int p = perm[s0 + k];
                    if (A.phase[p] != 0) continue;
                    const double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
                    AxisW<R, W> az;
                    p2g_axis_weights<R, ORD>(*tab, P, 2, dual_x(P, 2, x[2]), iv[2], inter[2], az);
                    const R wz = pick<W>(az.w, sz), dzw = pick<W>(az.dw, sz);
                    if (wz == R(0) && dzw == R(0)) continue;
                    any = true;
                    AxisW<R, W> ax, ay;
                    p2g_axis_weights<R, ORD>(*tab, P, 0, dual_x(P, 0, x[0]), iv[0], inter[0], ax);
                    p2g_axis_weights<R, ORD>(*tab, P, 1, dual_x(P, 1, x[1]), iv[1], inter[1], ay);
                    // every channel is deposited; the nodal kernel keeps
                    // the ones the call asked for
                    P2GCoef<R, THERM> q;
                    q.m = A.mass[p];
                    const R vol = A.vol[p];
                    const bool slab = P.external_loads && x[0] > P.slab_lo[0] && x[0] < P.slab_hi[0] &&
                                      x[1] > P.slab_lo[1] && x[1] < P.slab_hi[1] && x[2] > P.slab_lo[2] &&
                                      x[2] < P.slab_hi[2];
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        q.mv[d] = q.m * A.v[d][p];
                        q.b[d] = q.m * grav[d] + (slab ? (R)P.extforce[d] : R(0));
                    }
#pragma unroll
                    for (int c6 = 0; c6 < 6; ++c6) q.s[c6] = -vol * A.sig[c6][p];
                    if constexpr (THERM) {
                        q.mcp = q.m * A.cp[p];
                        q.mcpT = (R)(q.mcp * (A.T[p] - P.Tref));
                        q.mk = q.m * A.kc[p];
#pragma unroll
                        for (int d = 0; d < 3; ++d) q.qv[d] = vol * A.q[d][p];
                        q.VQ = vol * A.Q[p];
                    }
                    if constexpr (sizeof(R) == 4) {
                        const float2 cm = make_float2(q.m, q.mv[0]), cp = make_float2(q.mv[1], q.mv[2]);
                        const float2 cb = make_float2(q.b[0], q.b[1]);
                        const float2 cs0 = make_float2(q.s[0], q.s[1]), cs1 = make_float2(q.s[1], q.s[3]),
                                     cs2 = make_float2(q.s[2], q.s[4]);
                        const float2 wzz = make_float2(wz, wz), dzz = make_float2(dzw, dzw);
#pragma unroll
                        for (int r = 0; r < ROWS; ++r) {
                            const float2 wyy = make_float2(ay.w[sy0 + r], ay.w[sy0 + r]);
                            const float2 dyy = make_float2(ay.dw[sy0 + r], ay.dw[sy0 + r]);
                            const float2 wyz = __fmul2_rn(wyy, wzz), dyz = __fmul2_rn(dyy, wzz),
                                         wdz = __fmul2_rn(wyy, dzz);
#pragma unroll
                            for (int sx = 0; sx < W; ++sx) {
                                const float2 wxx = make_float2(ax.w[sx], ax.w[sx]);
                                const float2 dxx = make_float2(ax.dw[sx], ax.dw[sx]);
                                acc[r][sx].add2(cm, cp, cb, cs0, cs1, cs2, q, __fmul2_rn(wxx, wyz),
                                                __fmul2_rn(dxx, wyz), __fmul2_rn(wxx, dyz), __fmul2_rn(wxx, wdz));
                            }
                        }
                    } else {
#pragma unroll
                        for (int r = 0; r < ROWS; ++r) {
                            const R wy = ay.w[sy0 + r], dyw = ay.dw[sy0 + r];
                            const R wyz = wy * wz, dyz = dyw * wz, wdz = wy * dzw;
#pragma unroll
                            for (int sx = 0; sx < W; ++sx) {
                                const R wx = ax.w[sx];
                                acc[r][sx].add(q, wx * wyz, ax.dw[sx] * wyz, wx * dyz, wx * wdz);
                            }
                        }
                    }
                }
                if (!any) continue;
#pragma unroll
                for (int r = 0; r < ROWS; ++r)
#pragma unroll
                    for (int sx = 0; sx < W; ++sx) {
                        const int idx = ((lz + sz) * B + (ly + sy0 + r)) * B + (lx + sx);
#pragma unroll
                        for (int ch = 0; ch < NCH; ++ch)
                            fx_add_r<R>(acc_lo, acc_hi, ch * B3 + idx, acc[r][sx].get(ch), sc[ch]);
                    }
            }
        }
    }
    __syncthreads();
    fx_store<R>(acc_lo, acc_hi, NCH * B3, staging + (long long)w * stg_stride<R>((long long)NCH * B3));
    __syncthreads();
}

template <class R, int ORD, bool THERM>
__global__ void __launch_bounds__(P2GCfg<R, ORD, THERM>::THREADS, P2GCfg<R, ORD, THERM>::MINB)
    k_p2g_cell(Params P, Parts<R> A, const int *active, const int *start, const int *cell_start, const int32_t *perm,
               long long *staging, Ctl *ctl, int flags) {
    constexpr int NCH = THERM ? CH_ALL : CH_MOM_END;
    __shared__ int s_item;
    extern __shared__ __align__(16) unsigned char smraw[];
    SplineTables *tab = reinterpret_cast<SplineTables *>(smraw);
    const int B3 = P.B * P.B * P.B;
    unsigned *acc_lo = reinterpret_cast<unsigned *>(smraw + ((sizeof(SplineTables) + 15) & ~15));
    int *acc_hi = reinterpret_cast<int *>(acc_lo + NCH * B3 * fx_lo_words<R>());
    load_tables(tab);
    R sc[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c) sc[c] = (R)ctl->scale[c];
    (void)flags;  // every channel is deposited; the nodal kernel keeps the requested ones
    R grav[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) grav[d] = (R)P.gravity[d];
    const int nitems = ctl->n_active_tiles;
    for (;;) {
        // tiles are taken in turn from a device counter: blocks that drew
        // light tiles take more of them
        if (threadIdx.x == 0) s_item = atomicAdd(&ctl->next_p2g, 1);
        fx_zero<R>(acc_lo, acc_hi, NCH * B3);
        __syncthreads();
        const int w = s_item;
        if (w >= nitems) break;
        p2g_tile<R, ORD, THERM>(tab, acc_lo, acc_hi, P, A, active, start, cell_start, perm, staging, sc, grav, w);
    }
}

// ---------------------------------------------------------------- K2 factorized P2G
// Momentum P2G of uniform quadratic (nearest-node bins) and cubic (cells)
// B-splines with the deposit of deposit_onto_grid_momentum
// (mpm_particle_grid_ops.cpp:484-577) in factorized form.  With
// N = wx wy wz and grad N = (dwx wy wz, wx dwy wz, wx wy dwz), s_dj =
// -V sigma_dj and b_d = m g_d (+ f_ext,d inside the force slab):
//   m N          = wx (wy (m wz))
//   m v_d N      = wx (wy (m v_d wz))
//   f_d          = wx (wy A_d + dwy B_d) + dwx (wy C_d),
//   A_d = b_d wz + s_d2 dwz,  B_d = s_d1 wz,  C_d = s_d0 wz,
// so a node costs 4 packed FP32 FMAs and 2 scalar ones (10 FMAs in FP64)
// instead of forming N and grad N.  Tasks are (cell, z-slice, row group):
// the W x NPASS tasks of a cell sit in adjacent threads, read the cell's
// particles together (they stay in L1) and each accumulates ROWS rows of its
// slice in registers, then adds the cell's sums to the tile's fixed-point
// node block.  Every node's register sum runs over the cell's particles in
// storage order with the same expression whatever ROWS and the block size
// are, so all launch variants give bit-identical results.
template <class R, int ROWS>
struct FactRow;  // row terms (wy and dwy folded into the z-level terms)
template <int ROWS>
struct FactRow<float, ROWS> {
    float2 mp0, p12, a01, c01;
    float a2, c2;
};
template <int ROWS>
struct FactRow<double, ROWS> {
    double m, p[3], a[3], c[3];
};

template <class R>
struct FactAcc;
template <>
struct FactAcc<float> {
    float2 mp0, p12, f01;
    float f2;
    __device__ __forceinline__ void zero() {
        mp0 = p12 = f01 = make_float2(0.f, 0.f);
        f2 = 0.f;
    }
    // GRP 0: every channel; 1: mass and momentum; 2: force (the same
    // operations on each channel in every case)
    template <int GRP = 0>
    __device__ __forceinline__ void add(const FactRow<float, 1> &r, float2 wxx, float2 dxx) {
        if (GRP != 2) {
            mp0 = __ffma2_rn(wxx, r.mp0, mp0);
            p12 = __ffma2_rn(wxx, r.p12, p12);
        }
        if (GRP != 1) {
            f01 = __ffma2_rn(wxx, r.a01, f01);
            f01 = __ffma2_rn(dxx, r.c01, f01);
            f2 = fmaf(wxx.x, r.a2, f2);
            f2 = fmaf(dxx.x, r.c2, f2);
        }
    }
    __device__ __forceinline__ float get(int ch) const {
        switch (ch) {
            case CH_M: return mp0.x;
            case CH_P: return mp0.y;
            case CH_P + 1: return p12.x;
            case CH_P + 2: return p12.y;
            case CH_F: return f01.x;
            case CH_F + 1: return f01.y;
            default: return f2;
        }
    }
};
template <>
struct FactAcc<double> {
    double c[CH_MOM_END];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < CH_MOM_END; ++i) c[i] = 0.0;
    }
    template <int GRP = 0>
    __device__ __forceinline__ void add(const FactRow<double, 1> &r, double wx, double dwx) {
        if (GRP != 2) {
            c[CH_M] = fma(wx, r.m, c[CH_M]);
#pragma unroll
            for (int d = 0; d < 3; ++d) c[CH_P + d] = fma(wx, r.p[d], c[CH_P + d]);
        }
        if (GRP != 1) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                c[CH_F + d] = fma(wx, r.a[d], c[CH_F + d]);
                c[CH_F + d] = fma(dwx, r.c[d], c[CH_F + d]);
            }
        }
    }
    __device__ __forceinline__ double get(int ch) const { return c[ch]; }
};

// z-level terms of one particle for one node plane
template <class R>
struct FactZ {
    R m, p[3], a[3], b[3], c[3];
};

template <class R>
__device__ __forceinline__ FactRow<R, 1> fact_row(const FactZ<R> &z, R wy, R dwy) {
    FactRow<R, 1> r;
    if constexpr (sizeof(R) == 4) {
        const float2 wyy = make_float2(wy, wy), dyy = make_float2(dwy, dwy);
        r.mp0 = __fmul2_rn(wyy, make_float2(z.m, z.p[0]));
        r.p12 = __fmul2_rn(wyy, make_float2(z.p[1], z.p[2]));
        r.a01 = __ffma2_rn(dyy, make_float2(z.b[0], z.b[1]), __fmul2_rn(wyy, make_float2(z.a[0], z.a[1])));
        r.a2 = fmaf(dwy, z.b[2], wy * z.a[2]);
        r.c01 = __fmul2_rn(wyy, make_float2(z.c[0], z.c[1]));
        r.c2 = wy * z.c[2];
    } else {
        r.m = wy * z.m;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            r.p[d] = wy * z.p[d];
            r.a[d] = fma(dwy, z.b[d], wy * z.a[d]);
            r.c[d] = wy * z.c[d];
        }
    }
    return r;
}

// Weight and derivative of one slot (the task's z-slice): the interior piece
// of that slot alone, or the boundary-aware tables.  s is warp-uniform (the
// task mapping gives a warp one slice), so the switch does not diverge.
template <class R, int ORD>
__device__ __forceinline__ void slot_weight(const SplineTables &tab, const Params &P, int d, double x, int i,
                                            bool interior, R f, int s, R &w, R &dw) {
    const R dxinv = (R)P.dxi[d];
    if (interior) {
        if constexpr (sizeof(R) == 4) {
            slot_weight_f32(ORD, f, s, w, dw);
        } else if constexpr (ORD == 3) {
            const R o6 = (R)kOneBySix, t3 = (R)kTwoByThree, f3 = (R)kFourByThree;
            const R z = f + R(1 - s), z2 = z * z;
            switch (s) {
                case 0: w = fma(-o6, z2 * z, fma(R(1), z2, fma(R(-2), z, f3))); dw = fma(R(-0.5), z2, fma(R(2), z, R(-2))); break;
                case 1: w = fma(R(0.5), z2 * z, fma(R(-1), z2, fma(R(0), z, t3))); dw = fma(R(1.5), z2, fma(R(-2), z, R(0))); break;
                case 2: w = fma(R(-0.5), z2 * z, fma(R(-1), z2, fma(R(0), z, t3))); dw = fma(R(-1.5), z2, fma(R(-2), z, R(0))); break;
                default: w = fma(o6, z2 * z, fma(R(1), z2, fma(R(2), z, f3))); dw = fma(R(0.5), z2, fma(R(2), z, R(2))); break;
            }
        } else {
            const R z = f + R(1 - s);
            switch (s) {
                case 0: w = fma(R(0.5), z * z, fma(R(-1.5), z, R(1.125))); dw = z - R(1.5); break;
                case 1: w = fma(R(-1), z * z, fma(R(0), z, R(0.75))); dw = R(-2) * z; break;
                default: w = fma(R(0.5), z * z, fma(R(1.5), z, R(1.125))); dw = z + R(1.5); break;
            }
        }
        dw *= dxinv;
    } else {
        AxisW<R, P2GStc<ORD>::W> a;
        p2g_axis_weights<R, ORD>(tab, P, d, x, i, false, a);
        w = pick<P2GStc<ORD>::W>(a.w, s);
        dw = pick<P2GStc<ORD>::W>(a.dw, s);
    }
}

// Weights of all slots of one axis: interior pieces from the offset f, the
// tables elsewhere.
template <class R, int ORD>
__device__ __forceinline__ void fact_axis_weights(const SplineTables &tab, const Params &P, int d, double x, int i,
                                                  bool interior, R f, AxisW<R, P2GStc<ORD>::W> &a) {
    if (interior)
        interior_weights<R, ORD>(f, (R)P.dxi[d], a);
    else
        p2g_axis_weights<R, ORD>(tab, P, d, x, i, false, a);
}

// The particles ka..kb-1 of one cell (bin) into a task's accumulators: for
// each particle the z weight of the task's slice first (a zero slice weight
// and derivative skip it), then the x and y weights, the particle's
// z-factored terms, and per y row of the task a packed FMA per node and
// channel pair.  Returns whether any particle contributed.
template <class R, int ORD, int ROWS, int MAP, int GRP = 0>
__device__ __forceinline__ bool fact_deposit_cell(const SplineTables *tab, const Params &P, const Parts<R> &A,
                                                  const int32_t *perm, int s0, int ka, int kb, const int iv[3],
                                                  const bool inter[3], const double xo[3], int sz, int rg,
                                                  const R *grav, FactAcc<R> (&acc)[ROWS][P2GStc<ORD>::W]) {
    constexpr int W = P2GStc<ORD>::W;
    constexpr int NPASS = W / ROWS;
    bool any = false;
    for (int k = ka; k < kb; ++k) {
        const int p = perm[s0 + k];
        if (A.phase[p] != 0) continue;
        const double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
        double xw[3];
        R f[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            xw[d] = dual_x(P, d, x[d]);
            f[d] = (R)((xw[d] - xo[d]) * P.dxi[d]);
        }
        R wz, dwz;
        if (MAP == 0) {
            slot_weight<R, ORD>(*tab, P, 2, xw[2], iv[2], inter[2], f[2], sz, wz, dwz);
        } else {
            AxisW<R, W> az;
            fact_axis_weights<R, ORD>(*tab, P, 2, xw[2], iv[2], inter[2], f[2], az);
            wz = pick<W>(az.w, sz);
            dwz = pick<W>(az.dw, sz);
        }
        if (wz == R(0) && dwz == R(0)) continue;
        any = true;
        AxisW<R, W> ax, ay;
        fact_axis_weights<R, ORD>(*tab, P, 0, xw[0], iv[0], inter[0], f[0], ax);
        fact_axis_weights<R, ORD>(*tab, P, 1, xw[1], iv[1], inter[1], f[1], ay);
        const R m = A.mass[p], vol = A.vol[p];
        const bool slab = P.external_loads && x[0] > P.slab_lo[0] && x[0] < P.slab_hi[0] && x[1] > P.slab_lo[1] &&
                          x[1] < P.slab_hi[1] && x[2] > P.slab_lo[2] && x[2] < P.slab_hi[2];
        R sg[6];
#pragma unroll
        for (int c6 = 0; c6 < 6; ++c6) sg[c6] = -vol * A.sig[c6][p];
        // rows of the symmetric stress in packed XX XY XZ YY YZ ZZ order
        const R s0r[3] = {sg[0], sg[1], sg[2]}, s1r[3] = {sg[1], sg[3], sg[4]}, s2r[3] = {sg[2], sg[4], sg[5]};
        FactZ<R> z;
        z.m = m * wz;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const R bd = fma(m, grav[d], slab ? (R)P.extforce[d] : R(0));
            const R sd0 = d == 0 ? s0r[0] : (d == 1 ? s1r[0] : s2r[0]);
            const R sd1 = d == 0 ? s0r[1] : (d == 1 ? s1r[1] : s2r[1]);
            const R sd2 = d == 0 ? s0r[2] : (d == 1 ? s1r[2] : s2r[2]);
            z.p[d] = (m * A.v[d][p]) * wz;
            z.a[d] = fma(sd2, dwz, bd * wz);
            z.b[d] = sd1 * wz;
            z.c[d] = sd0 * wz;
        }
#pragma unroll
        for (int r = 0; r < ROWS; ++r) {
            const int sy = rg * ROWS + r;
            const R wy = NPASS == 1 ? ay.w[r] : pick<W>(ay.w, sy);
            const R dwy = NPASS == 1 ? ay.dw[r] : pick<W>(ay.dw, sy);
            const FactRow<R, 1> row = fact_row<R>(z, wy, dwy);
#pragma unroll
            for (int sx = 0; sx < W; ++sx) {
                if constexpr (sizeof(R) == 4)
                    acc[r][sx].template add<GRP>(row, make_float2(ax.w[sx], ax.w[sx]),
                                                 make_float2(ax.dw[sx], ax.dw[sx]));
                else
                    acc[r][sx].template add<GRP>(row, ax.w[sx], ax.dw[sx]);
            }
        }
    }
    return any;
}

// L2 prefetch of the first particle of cell c, if it has one.
template <class R>
__device__ __forceinline__ void prefetch_cell_head(const Parts<R> &A, const int32_t *perm, int s0, const int *cs,
                                                   int c) {
    const int kn = cs[c];
    if (kn < cs[c + 1]) {
        const int pn = perm[s0 + kn];
        auto pf = [](const void *q) { asm volatile("prefetch.global.L2 [%0];" ::"l"(q)); };
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            pf(A.x[d] + pn);
            pf(A.v[d] + pn);
        }
#pragma unroll
        for (int c6 = 0; c6 < 6; ++c6) pf(A.sig[c6] + pn);
        pf(A.mass + pn);
        pf(A.vol + pn);
        pf(A.phase + pn);
    }
}

template <class R, int ORD>
__device__ __forceinline__ void cell_frame(const Params &P, const int tc[3], int lx, int ly, int lz, int iv[3],
                                           bool inter[3], double xo[3]) {
    const int T = P.T;
    iv[0] = tc[0] * T + lx;
    iv[1] = tc[1] * T + ly;
    iv[2] = tc[2] * T + lz;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        inter[d] = P.periodic[d] ||
                   (ORD == 2 ? (iv[d] >= 3 && iv[d] <= P.nc[d] - 3) : (iv[d] >= 3 && iv[d] <= P.nc[d] - 4));
        xo[d] = P.plo[d] + iv[d] * P.dx[d];  // the cell's (cubic) or bin node's (quadratic) coordinate
    }
}

// One tile of the factorized P2G, one task per (cell, z-slice, row group,
// channel group): the task's ROWS x W node block accumulates the cell's
// particles in registers and is added to the tile's fixed-point block after
// the cell.  With GROUPS = 2 a cell's mass and momentum (4 channels, no
// gradients, no stress) and its force (3 channels) go to separate tasks:
// each holds at most 64 accumulators instead of 112, so two blocks fit an
// SM, for about the same instructions; each channel's operations are the
// same as with GROUPS = 1, so the results are the same bits.
template <class R, int ORD, int ROWS, int MAP, int GROUPS = 1>
__device__ __forceinline__ void p2g_tile_fact(const SplineTables *tab, unsigned *acc_lo, int *acc_hi, const Params &P,
                                              const Parts<R> &A, const int *active, const int *start,
                                              const int *cell_start, const int32_t *perm, long long *staging,
                                              const R *sc, const R *grav, int w) {
    constexpr int W = P2GStc<ORD>::W;
    static_assert(W % ROWS == 0, "rows per pass must divide the stencil width");
    constexpr int NPASS = W / ROWS, LANES = W * NPASS * GROUPS, NCH = CH_MOM_END;
    const int B = P.B, B3 = B * B * B, T = P.T, T3 = T * T * T;
    const int t = active[w];
    int tc[3];
    tile_coords(P, t, tc);
    const int s0 = start[t];
    const int *cs = cell_start + (long long)w * (T3 + 1);
    // The tile's non-empty cells, in cell order (a block-wide compaction), so
    // that no lane walks an empty cell: at a body's surface half the cells
    // of a tile can be empty.  Cells keep their own sums, and the fixed-point
    // adds do not depend on the order, so the results do not change.
    __shared__ int s_cells[kMaxTileCells];
    __shared__ int s_scan[34];
    int ncomp;
    {
        const int per = (T3 + (int)blockDim.x - 1) / (int)blockDim.x, c0 = (int)threadIdx.x * per;
        int cnt = 0;
        for (int k = 0; k < per; ++k) {
            const int cc = c0 + k;
            cnt += (cc < T3 && cs[cc] < cs[cc + 1]) ? 1 : 0;
        }
        int off = block_exclusive_scan(cnt, &ncomp, s_scan);
        for (int k = 0; k < per; ++k) {
            const int cc = c0 + k;
            if (cc < T3 && cs[cc] < cs[cc + 1]) s_cells[off++] = cc;
        }
        __syncthreads();
    }
    // task u -> (cell index in the compacted list, sub) with sub = (z-slice,
    // row group, channel group).  MAP 0: warp u / 32 takes one sub of 32
    // consecutive listed cells, so the slice and the channel group are
    // warp-uniform (one z weight evaluated, no divergence); the LANES warps
    // of a group of 32 cells are consecutive and run together (the cells'
    // particles stay in L1).  MAP 1: a cell's LANES tasks sit in adjacent
    // lanes, which read each particle with one load.
    const int nlist = MAP == 0 ? ((ncomp + 31) & ~31) : ncomp;
    const int ntask = LANES * nlist, step = (int)blockDim.x;
    auto task = [&](int uu, int &cc, int &ss) {
        if (MAP == 0) {
            const int wi = uu >> 5, g = wi / LANES;
            ss = wi - g * LANES;
            cc = g * 32 + (uu & 31);
        } else {
            cc = uu / LANES;
            ss = uu - cc * LANES;
        }
    };
    for (int u = threadIdx.x; u < ntask; u += step) {
        int ci, sub;
        task(u, ci, sub);
        if (ci >= ncomp) continue;
        const int c = s_cells[ci];
        const int grp = GROUPS == 1 ? 0 : sub % GROUPS, sp = sub / GROUPS;
        const int sz = sp / NPASS, rg = sp - sz * NPASS;
        const int ka = cs[c], kb = cs[c + 1];
        if (EXG_P2G_PREFETCH && sub == 0) {
            // L2 prefetch of the first particle of the cell this thread takes next
            const int un = u + step;
            int cn = 0, sn = 1;
            if (un < ntask) task(un, cn, sn);
            if (un < ntask && sn == 0 && cn < ncomp) prefetch_cell_head(A, perm, s0, cs, s_cells[cn]);
        }
        const int lx = c % T, ly = (c / T) % T, lz = c / (T * T);
        int iv[3];
        bool inter[3];
        double xo[3];
        cell_frame<R, ORD>(P, tc, lx, ly, lz, iv, inter, xo);
        // each branch has its own accumulators (only its channels live)
        auto cell_task = [&](auto grp_tag) {
            constexpr int G = decltype(grp_tag)::value;
            constexpr int CH0 = G == 2 ? CH_F : 0, CH1 = G == 1 ? CH_F : NCH;
            FactAcc<R> acc[ROWS][W];
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
#pragma unroll
                for (int sx = 0; sx < W; ++sx) acc[r][sx].zero();
            if (!fact_deposit_cell<R, ORD, ROWS, MAP, G>(tab, P, A, perm, s0, ka, kb, iv, inter, xo, sz, rg, grav,
                                                         acc))
                return;
#pragma unroll
            for (int r = 0; r < ROWS; ++r)
#pragma unroll
                for (int sx = 0; sx < W; ++sx) {
                    const int idx = ((lz + sz) * B + (ly + rg * ROWS + r)) * B + (lx + sx);
#pragma unroll
                    for (int ch = CH0; ch < CH1; ++ch)
                        fx_add_r<R>(acc_lo, acc_hi, ch * B3 + idx, acc[r][sx].get(ch), sc[ch]);
                }
        };
        if (GROUPS == 1)
            cell_task(std::integral_constant<int, 0>{});
        else if (grp == 0)
            cell_task(std::integral_constant<int, 1>{});
        else
            cell_task(std::integral_constant<int, 2>{});
    }
    __syncthreads();
    fx_store<R>(acc_lo, acc_hi, NCH * B3, staging + (long long)w * stg_stride<R>((long long)NCH * B3));
    __syncthreads();
}

// Segments a row of a tile is cut into for p2g_tile_xrun (1: whole rows;
// half rows measured no faster: the block's closing barrier waits for the
// slowest segment either way).
constexpr int kXRunParts = 1;

// One tile of the factorized P2G, one task per (segment of T / kXRunParts
// cells along x, z-slice, row group): the task walks its segment's cells in
// x order with a window of W node columns in registers.  Once cell cx is
// done, no later cell of the segment reaches node column cx, so that column
// alone goes to the tile's fixed-point block and the window moves by one
// column; the last W - 1 columns go after the segment.  Per cell one column
// of ROWS x 7 values is converted and added instead of W columns.
template <class R, int ORD, int ROWS, int MAP>
__device__ __forceinline__ void p2g_tile_xrun(const SplineTables *tab, unsigned *acc_lo, int *acc_hi, const Params &P,
                                              const Parts<R> &A, const int *active, const int *start,
                                              const int *cell_start, const int32_t *perm, long long *staging,
                                              const R *sc, const R *grav, int w) {
    constexpr int W = P2GStc<ORD>::W;
    static_assert(W % ROWS == 0, "rows per pass must divide the stencil width");
    constexpr int NPASS = W / ROWS, LANES = W * NPASS, NCH = CH_MOM_END;
    const int B = P.B, B3 = B * B * B, T = P.T, T2 = T * T, T3 = T2 * T;
    const int SL = T / kXRunParts, NSEG = T2 * kXRunParts;  // cells per segment, segments per tile
    const int t = active[w];
    int tc[3];
    tile_coords(P, t, tc);
    const int s0 = start[t];
    const int *cs = cell_start + (long long)w * (T3 + 1);
    // task u -> (segment, z-slice, row group); MAP 0: a warp takes one
    // (z-slice, row group) of 32 segments (warp-uniform slice), MAP 1: a
    // segment's LANES tasks in adjacent lanes
    const int groups = (NSEG + 31) >> 5;
    const int ntask = MAP == 0 ? groups * 32 * LANES : NSEG * LANES, step = (int)blockDim.x;
    for (int u = threadIdx.x; u < ntask; u += step) {
        int seg, sub;
        if (MAP == 0) {
            const int wi = u >> 5, g = wi / LANES;
            sub = wi - g * LANES;
            seg = g * 32 + (u & 31);
        } else {
            seg = u / LANES;
            sub = u - seg * LANES;
        }
        if (seg >= NSEG) continue;
        const int sz = sub / NPASS, rg = sub - sz * NPASS;
        const int row = seg / kXRunParts, x0 = (seg - row * kXRunParts) * SL;
        const int ly = row % T, lz = row / T;
        const int c0 = row * T + x0;  // first cell of the segment (x fastest)
        FactAcc<R> acc[ROWS][W];
#pragma unroll
        for (int r = 0; r < ROWS; ++r)
#pragma unroll
            for (int sx = 0; sx < W; ++sx) acc[r][sx].zero();
        unsigned dirty = 0;  // bit j: window column j holds contributions
        const int ybase = (lz + sz) * B + ly + rg * ROWS;
        auto flush = [&](int j, int col) {
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
                const int idx = (ybase + r) * B + col;
#pragma unroll
                for (int ch = 0; ch < NCH; ++ch) {
                    R v;
                    switch (j) {  // j is a compile-time constant at every call
                        case 0: v = acc[r][0].get(ch); break;
                        case 1: v = acc[r][1 % W].get(ch); break;
                        case 2: v = acc[r][2 % W].get(ch); break;
                        default: v = acc[r][W - 1].get(ch); break;
                    }
                    fx_add_r<R>(acc_lo, acc_hi, ch * B3 + idx, v, sc[ch]);
                }
            }
        };
        for (int k = 0; k < SL; ++k) {
            const int cx = x0 + k, c = c0 + k;
            const int ka = cs[c], kb = cs[c + 1];
            if (EXG_P2G_PREFETCH && k + 1 < SL && sub == 0) prefetch_cell_head(A, perm, s0, cs, c + 1);
            if (ka < kb) {
                int iv[3];
                bool inter[3];
                double xo[3];
                cell_frame<R, ORD>(P, tc, cx, ly, lz, iv, inter, xo);
                if (fact_deposit_cell<R, ORD, ROWS, MAP>(tab, P, A, perm, s0, ka, kb, iv, inter, xo, sz, rg, grav,
                                                         acc))
                    dirty |= (1u << W) - 1u;
            }
            if (dirty & 1u) flush(0, cx);
            // the window moves one column along x
#pragma unroll
            for (int r = 0; r < ROWS; ++r) {
#pragma unroll
                for (int j = 0; j + 1 < W; ++j) acc[r][j] = acc[r][j + 1];
                acc[r][W - 1].zero();
            }
            dirty >>= 1;
        }
#pragma unroll
        for (int j = 0; j + 1 < W; ++j)
            if (dirty & (1u << j)) flush(j, x0 + SL + j);
    }
    __syncthreads();
    fx_store<R>(acc_lo, acc_hi, NCH * B3, staging + (long long)w * stg_stride<R>((long long)NCH * B3));
    __syncthreads();
}

// FP64 cubic tasks walk rows of cells (p2g_tile_xrun): its fixed-point
// adds are returning 64-bit atomics, and the walk converts and adds a third
// as many values (FP64 P2G 3.46 -> 2.97 ms on the 9 M-particle spheres).
// FP32 cubic and all quadratic tasks take one cell (bin) each
// (p2g_tile_fact): the FP32 adds are cheap, and the per-cell walk keeps
// more tasks per thread to even out uneven cells (1.66 against 1.69 ms).
// Every launch variant of one precision and order uses the same walk, so
// the register sums and hence the results are the same for all of them.
template <class R, int ORD, int ROWS, int MAP, int GROUPS = 1>
__device__ __forceinline__ void p2g_tile_factorized(const SplineTables *tab, unsigned *acc_lo, int *acc_hi,
                                                    const Params &P, const Parts<R> &A, const int *active,
                                                    const int *start, const int *cell_start, const int32_t *perm,
                                                    long long *staging, const R *sc, const R *grav, int w) {
    if constexpr (ORD == 3 && sizeof(R) == 8)
        p2g_tile_xrun<R, ORD, ROWS, MAP>(tab, acc_lo, acc_hi, P, A, active, start, cell_start, perm, staging, sc,
                                         grav, w);
    else
        p2g_tile_fact<R, ORD, ROWS, MAP, GROUPS>(tab, acc_lo, acc_hi, P, A, active, start, cell_start, perm,
                                                 staging, sc, grav, w);
}

template <class R, int ORD, int V>
__global__ void __launch_bounds__(P2GVar<R, ORD, V>::THREADS, P2GVar<R, ORD, V>::MINB)
    k_p2g_fact(Params P, Parts<R> A, const int *active, const int *start, const int *cell_start, const int32_t *perm,
               long long *staging, Ctl *ctl) {
    constexpr int NCH = CH_MOM_END;
    __shared__ int s_item;
    extern __shared__ __align__(16) unsigned char smraw[];
    SplineTables *tab = reinterpret_cast<SplineTables *>(smraw);
    const int B3 = P.B * P.B * P.B;
    unsigned *acc_lo = reinterpret_cast<unsigned *>(smraw + ((sizeof(SplineTables) + 15) & ~15));
    int *acc_hi = reinterpret_cast<int *>(acc_lo + NCH * B3 * fx_lo_words<R>());
    load_tables(tab);
    R sc[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c) sc[c] = (R)ctl->scale[c];
    R grav[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) grav[d] = (R)P.gravity[d];
    const int nitems = ctl->n_active_tiles;
    for (;;) {
        // tiles are taken in turn from a device counter
        if (threadIdx.x == 0) s_item = atomicAdd(&ctl->next_p2g, 1);
        fx_zero<R>(acc_lo, acc_hi, NCH * B3);
        __syncthreads();
        const int w = s_item;
        if (w >= nitems) break;
        p2g_tile_factorized<R, ORD, P2GVar<R, ORD, V>::ROWS, P2GVar<R, ORD, V>::MAP, P2GVar<R, ORD, V>::GROUPS>(
            tab, acc_lo, acc_hi, P, A, active, start, cell_start, perm, staging, sc, grav, w);
    }
}

// Domain-wall BCs of one node (nodal_bcs, nodal_data_ops.cpp:663-766),
// UDF walls (apply_udf_nodal_bcs, :1061-1175) and level-set bodies
// (nodal_levelset_bcs, :129-220).  v is updated in place.
struct NodeBCArgs {
    const double *udf[2][3];
    const double *ls[kMaxBodies];
    const double *udfT[2][3];  // wall-temperature tables: (value, second value) per face node
};

__device__ __forceinline__ double ls_node_value(const Params &P, const double *phi, int i, int j, int k) {
    int id[3] = {i, j, k};
    for (int d = 0; d < 3; ++d) {
        if (P.periodic[d]) {
            int n = P.nc[d];
            id[d] %= n;
            if (id[d] < 0) id[d] += n;
        } else if (id[d] < 0 || id[d] > P.nc[d]) {
            return 1.0;
        }
    }
    return phi[((long long)id[2] * P.nn[1] + id[1]) * P.nn[0] + id[0]];
}

// get_levelset_value / get_levelset_grad (Source/mpm_eb.H:176-288), lsref 1.
__device__ void ls_sample(const Params &P, const double *phi, const double x[3], double &val, double g[3]) {
    int idx[3];
    for (int d = 0; d < 3; ++d) idx[d] = (int)floor((x[d] - P.plo[d] + kTiny) / P.dx[d]);
    double dv[3][2], w[3][2];
    for (int d = 0; d < 3; ++d) {
        double r = (x[d] - (P.plo[d] + idx[d] * P.dx[d])) / P.dx[d];
        w[d][0] = 1.0 - r;
        w[d][1] = r;
        dv[d][0] = -(1.0 / P.dx[d]);
        dv[d][1] = 1.0 / P.dx[d];
    }
    val = 0.0;
    g[0] = g[1] = g[2] = 0.0;
    for (int corner = 0; corner < 8; ++corner) {
        int o[3], c[3];
        for (int d = 0; d < 3; ++d) {
            o[d] = (corner >> d) & 1;
            c[d] = min(max(idx[d] + o[d], -1), P.nc[d] + 1);
        }
        double ph = ls_node_value(P, phi, c[0], c[1], c[2]);
        double bv = w[0][o[0]] * w[1][o[1]] * w[2][o[2]];
        val += ph * bv;
        g[0] += ph * (dv[0][o[0]] * w[1][o[1]] * w[2][o[2]]);
        g[1] += ph * (w[0][o[0]] * dv[1][o[1]] * w[2][o[2]]);
        g[2] += ph * (w[0][o[0]] * w[1][o[1]] * dv[2][o[2]]);
    }
}

// Domain walls of one node (nodal_bcs): relvel_in accumulates the wall
// velocity of each face the node lies on; relvel_out persists across
// directions.
__device__ __forceinline__ void node_wall_bcs(const Params &P, int i, int j, int k, double v[3], unsigned &status) {
    const int id[3] = {i, j, k};
    double rin[3] = {v[0], v[1], v[2]}, rout[3] = {v[0], v[1], v[2]};
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
        const bool lo = id[dir] == 0;
        const bool hi = !lo && id[dir] == P.nc[dir];
        if (!lo && !hi) continue;
        double wv[3];
        for (int d = 0; d < 3; ++d) {
            wv[d] = lo ? P.wvel_lo[dir * 3 + d] : P.wvel_hi[dir * 3 + d];
            rin[d] -= wv[d];
        }
        double nd[3] = {0, 0, 0};
        nd[dir] = lo ? 1.0 : -1.0;
        if (applybc<double>(rin, rout, lo ? P.wmu_lo[dir] : P.wmu_hi[dir], nd, lo ? P.bclo[dir] : P.bchi[dir]) < 0)
            status |= ST_BC;
        for (int c = 0; c < 3; ++c) v[c] = rout[c] + wv[c];
    }
}

__device__ void node_bcs(const Params &P, const NodeBCArgs &bc, int i, int j, int k, double m, double v[3],
                         unsigned &status) {
    const int id[3] = {i, j, k};
    node_wall_bcs(P, i, j, k, v, status);
    // UDF wall velocity tables
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
        const double *tab = nullptr;
        int bct = -1;
        if (id[dir] == 0 && bc.udf[0][dir]) {
            tab = bc.udf[0][dir];
            bct = P.bclo[dir];
        } else if (id[dir] == P.nc[dir] && bc.udf[1][dir]) {
            tab = bc.udf[1][dir];
            bct = P.bchi[dir];
        }
        if (!tab) continue;
        const int p0 = (dir == 0) ? 1 : 0, p1 = (dir == 2) ? 1 : 2;
        const long long f = ((long long)id[p0] * (P.nc[p1] + 1) + id[p1]) * 3;
        if (bct == EXG_BC_NOSLIP) {
            for (int c = 0; c < 3; ++c) v[c] = tab[f + c];
        } else {
            v[dir] = tab[f + dir];
        }
    }
    // level-set bodies
    if (P.num_bodies > 0 && m > 0.0) {
        const double xn[3] = {P.plo[0] + i * P.dx[0], P.plo[1] + j * P.dx[1], P.plo[2] + k * P.dx[2]};
        for (int b = 0; b < P.num_bodies; ++b) {
            if (!bc.ls[b]) continue;
            double lv, nd[3];
            ls_sample(P, bc.ls[b], xn, lv, nd);
            if (lv >= 0.0) continue;
            double gm = sqrt(nd[0] * nd[0] + nd[1] * nd[1] + nd[2] * nd[2]);
            if (!(gm >= 1.0e-10)) continue;
            for (int d = 0; d < 3; ++d) nd[d] /= gm;
            const Body &bd = P.body[b];
            double rin[3], rout[3];
            for (int d = 0; d < 3; ++d) {
                rin[d] = v[d] - bd.wall_vel[d];
                rout[d] = rin[d];
            }
            double veln = rin[0] * nd[0] + rin[1] * nd[1] + rin[2] * nd[2];
            if (veln > 0.0) continue;
            if (applybc<double>(rin, rout, bd.wall_mu, nd, bd.mom_bc) < 0) status |= ST_BC;
            for (int d = 0; d < 3; ++d) v[d] = rout[d] + bd.wall_vel[d];
        }
    }
}

// One node's record for the fused G2P: v and dv rounded to R as the dense
// arrays hold them, in the layout of the G2P's shared-memory node block.
template <class R>
__device__ __forceinline__ void write_rec(R *rec, long long ni, const double v[3], const double dv[3]) {
    if constexpr (sizeof(R) == 4) {
        float *q = rec + ni * 8;
        *reinterpret_cast<float4 *>(q) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)dv[0]);
        *reinterpret_cast<float4 *>(q + 4) = make_float4((float)dv[1], (float)dv[2], 0.f, 0.f);
    } else {
        double *q = rec + ni * 6;
        *reinterpret_cast<double2 *>(q) = make_double2(v[0], v[1]);
        *reinterpret_cast<double2 *>(q + 2) = make_double2(v[2], dv[0]);
        *reinterpret_cast<double2 *>(q + 4) = make_double2(dv[1], dv[2]);
    }
}

// ---------------------------------------------------------------- K3 nodes
// One CTA per tile; each thread owns nodes of the tile, adds the fixed-point
// partials of the <= 8 node blocks covering the node (exact integer sums),
// converts to FP64 and applies the nodal operations of the mode.
// One tile of the nodal kernel: every owned node of tile tiles[w] (or w).
template <class R, bool THERM, bool LEAN = false>
__device__ __forceinline__ void nodes_tile(const Params &P, const Nodes<R> &Nd, const NodeBCArgs &bc, const int *tiles,
                                           const int *slot, const long long *staging, const double *isc, double dt,
                                           int mode, int flags, int w, unsigned &status) {
    constexpr int NCH = THERM ? CH_ALL : CH_MOM_END;
    const int B = P.B, B3 = B * B * B, T = P.T;
    const int t = tiles ? tiles[w] : w;
    int tc[3];
    tile_coords(P, t, tc);
    for (int ln = threadIdx.x; ln < T * T * T; ln += blockDim.x) {
        const int l[3] = {ln % T, (ln / T) % T, ln / (T * T)};
        int nid[3];
        bool ok = true;
        for (int d = 0; d < 3; ++d) {
            nid[d] = tc[d] * T + l[d];
            const int nown = P.periodic[d] ? P.nc[d] : P.nc[d] + 1;
            ok = ok && nid[d] < nown;
        }
        if (!ok) continue;
        FxSum<R> accv[NCH];
#pragma unroll
        for (int c = 0; c < NCH; ++c) accv[c] = FxSum<R>();
        // Source tiles per axis: the node's own tile, plus the lower
        // neighbour when the node lies in its high halo (l < hhi) or the
        // upper neighbour when it lies in its low halo (l >= T - hlo); both
        // cannot happen since hhi + hlo <= T.
        int s1[3], l1[3], s2[3], l2[3];
        bool h2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s1[d] = tc[d];
            l1[d] = l[d] + P.hlo;
            h2[d] = true;
            if (l[d] < P.hhi) {
                s2[d] = tc[d] - 1;
                l2[d] = l[d] + P.hlo + T;
            } else if (l[d] >= T - P.hlo) {
                s2[d] = tc[d] + 1;
                l2[d] = l[d] + P.hlo - T;
            } else {
                s2[d] = 0;
                l2[d] = 0;
                h2[d] = false;
            }
            if (h2[d] && (s2[d] < 0 || s2[d] >= P.ntile[d])) {
                if (P.periodic[d])
                    s2[d] = (s2[d] + P.ntile[d]) % P.ntile[d];
                else
                    h2[d] = false;
            }
        }
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b2 = 0; b2 < 2; ++b2)
#pragma unroll
                for (int c2 = 0; c2 < 2; ++c2) {
                    if ((a && !h2[2]) || (b2 && !h2[1]) || (c2 && !h2[0])) continue;
                    const int sz = a ? s2[2] : s1[2], sy = b2 ? s2[1] : s1[1], sx = c2 ? s2[0] : s1[0];
                    const int lz = a ? l2[2] : l1[2], ly = b2 ? l2[1] : l1[1], lx = c2 ? l2[0] : l1[0];
                    const int sl = slot[(sz * P.ntile[1] + sy) * P.ntile[0] + sx];
                    if (sl < 0) continue;
                    const long long nv = (long long)NCH * B3;
                    const long long *blk = staging + (long long)sl * stg_stride<R>(nv);
                    const long long off = ((long long)lz * B + ly) * B + lx;
#pragma unroll
                    for (int c = 0; c < NCH; ++c) accv[c].add(blk, nv, off + (long long)c * B3);
                }
        const long long ni = ((long long)nid[2] * P.nn[1] + nid[1]) * P.nn[0] + nid[0];
        double m = accv[CH_M].value() * isc[CH_M];
        double p[3], f[3];
        for (int d = 0; d < 3; ++d) {
            p[d] = accv[CH_P + d].value() * isc[CH_P + d];
            f[d] = accv[CH_F + d].value() * isc[CH_F + d];
        }
        if (mode == NM_MERGE) {
            // P2G_Momentum: zero + deposit + normalise (mpm_particle_grid_ops.cpp:368-627)
            if (flags & PF_MASS)
                Nd.c[EXG_N_MASS][ni] = (R)m;
            else
                m = (double)Nd.c[EXG_N_MASS][ni];
            if (flags & PF_VEL) {
                double v[3] = {p[0], p[1], p[2]};
                if (m > 0.0)
                    for (int d = 0; d < 3; ++d) v[d] = (m >= P.mass_tol) ? p[d] / m : 0.0;
                for (int d = 0; d < 3; ++d) Nd.c[EXG_N_VEL + d][ni] = (R)v[d];
            }
            if (flags & PF_FORCE)
                for (int d = 0; d < 3; ++d) Nd.c[EXG_N_FRC + d][ni] = (R)f[d];
            if (THERM && (flags & (PF_TEMP | PF_SRC))) {
                // P2G_Temperature with reset: m cp, m cp T and the source are
                // zeroed, m k only when temperatures are deposited, and T is
                // normalised where m cp > 0 (mpm_particle_grid_ops.cpp:680-884)
                const bool fT = flags & PF_TEMP;
                const double mc = fT ? accv[CH_MC].value() * isc[CH_MC] : 0.0;
                const double mct = fT ? accv[CH_MCT].value() * isc[CH_MCT] : 0.0;
                Nd.c[EXG_N_MASS_SPHEAT][ni] = (R)mc;
                Nd.c[EXG_N_MASS_SPHEAT_TEMP][ni] = (R)mct;
                Nd.c[EXG_N_SOURCE_TEMP][ni] = (R)((flags & PF_SRC) ? accv[CH_SRC].value() * isc[CH_SRC] : 0.0);
                if (fT) {
                    Nd.c[EXG_N_MASS_COND][ni] = (R)(accv[CH_MK].value() * isc[CH_MK]);
                    if (mc > 0.0) Nd.c[EXG_N_TEMPERATURE][ni] = (R)((mc >= P.mass_tol) ? mct / mc : -P.Tref);
                }
            }
        } else if (mode == NM_FUSED) {
            double v[3] = {p[0], p[1], p[2]};
            if (m > 0.0)
                for (int d = 0; d < 3; ++d) v[d] = (m >= P.mass_tol) ? p[d] / m : 0.0;
            double vold[3] = {0, 0, 0}, mold = 0.0;
            if (m > 0.0) {  // backup_current_velocity
                mold = m;
                for (int d = 0; d < 3; ++d) vold[d] = v[d];
            }
            if (m >= P.mass_tol)  // Nodal_Time_Update_Momentum
                for (int d = 0; d < 3; ++d) v[d] += f[d] / m * dt;
            else
                v[0] = v[1] = v[2] = 0.0;
            if (LEAN)
                node_wall_bcs(P, nid[0], nid[1], nid[2], v, status);
            else
                node_bcs(P, bc, nid[0], nid[1], nid[2], m, v, status);
            double dv[3] = {0, 0, 0};
            if (m > 0.0)  // store_delta_velocity
                for (int d = 0; d < 3; ++d) dv[d] = v[d] - vold[d];
            Nd.c[EXG_N_MASS][ni] = (R)m;
            Nd.c[EXG_N_MASS_OLD][ni] = (R)mold;
            for (int d = 0; d < 3; ++d) {
                Nd.c[EXG_N_VEL + d][ni] = (R)v[d];
                Nd.c[EXG_N_FRC + d][ni] = (R)f[d];
                Nd.c[EXG_N_DVEL + d][ni] = (R)dv[d];
            }
            if (Nd.rec) write_rec<R>(Nd.rec, ni, v, dv);
            if (THERM && (flags & PF_TEMP)) {
                // P2G_Temperature(1,1,1), backup_current_temperature and
                // Nodal_Time_Update_Temperature (main.cpp:100-102) on a node
                // that Reset_Nodaldata_to_Zero left at 0
                const double mc = accv[CH_MC].value() * isc[CH_MC], mct = accv[CH_MCT].value() * isc[CH_MCT];
                const double src = accv[CH_SRC].value() * isc[CH_SRC];
                // temperatures relative to Tref (0 K is -Tref); DELTA holds 0
                // where m cp = 0, as the reset leaves it
                double Tn = -P.Tref;
                if (mc > 0.0) Tn = (mc >= P.mass_tol) ? mct / mc : -P.Tref;
                const double Told = (mc > 0.0) ? Tn : 0.0;
                if (mc >= P.mass_tol)
                    Tn += src / mc * dt;
                else
                    Tn = -P.Tref;
                Nd.c[EXG_N_MASS_SPHEAT][ni] = (R)mc;
                Nd.c[EXG_N_MASS_SPHEAT_TEMP][ni] = (R)mct;
                Nd.c[EXG_N_MASS_COND][ni] = (R)(accv[CH_MK].value() * isc[CH_MK]);
                Nd.c[EXG_N_SOURCE_TEMP][ni] = (R)src;
                Nd.c[EXG_N_TEMPERATURE][ni] = (R)Tn;
                Nd.c[EXG_N_DELTA_TEMPERATURE][ni] = (R)Told;
            }
        } else {  // NM_MUSL2: P2G(0,1,0) + Apply_Nodal_BCs (main.cpp:124-127)
            m = (double)Nd.c[EXG_N_MASS][ni];
            double v[3] = {p[0], p[1], p[2]};
            if (m > 0.0)
                for (int d = 0; d < 3; ++d) v[d] = (m >= P.mass_tol) ? p[d] / m : 0.0;
            if (LEAN)
                node_wall_bcs(P, nid[0], nid[1], nid[2], v, status);
            else
                node_bcs(P, bc, nid[0], nid[1], nid[2], m, v, status);
            double dv[3];
            for (int d = 0; d < 3; ++d) {
                Nd.c[EXG_N_VEL + d][ni] = (R)v[d];
                const R dold = Nd.c[EXG_N_DVEL + d][ni];
                const R dnew = (m > 0.0) ? (R)(v[d] - (double)dold) : dold;
                if (m > 0.0) Nd.c[EXG_N_DVEL + d][ni] = dnew;
                dv[d] = (double)dnew;
            }
            if (Nd.rec) write_rec<R>(Nd.rec, ni, v, dv);
            if (THERM && (flags & PF_SRC)) {
                // P2G_Temperature(1,0,1) of MUSL (main.cpp:133): the reset
                // zeroes m cp and m cp T, only the source is deposited
                Nd.c[EXG_N_MASS_SPHEAT][ni] = R(0);
                Nd.c[EXG_N_MASS_SPHEAT_TEMP][ni] = R(0);
                Nd.c[EXG_N_SOURCE_TEMP][ni] = (R)(accv[CH_SRC].value() * isc[CH_SRC]);
            }
        }
    }
}

// Four 256-thread blocks per SM (64 registers, some spilled): the per-node
// work is a chain of dependent loads (slot, then up to eight staging
// blocks), so occupancy decides its speed (the dam break's nodal update
// 0.171 ms with one block per SM and no register cap, 0.108 / 0.086 / 0.080
// ms with two / three / four blocks)
#ifndef EXG_NODES_MINB
#define EXG_NODES_MINB 4
#endif
template <class R, bool THERM, bool LEAN = false>
__global__ void __launch_bounds__(kThreads, EXG_NODES_MINB) k_nodes(Params P, Nodes<R> Nd, NodeBCArgs bc, const int *tiles,
                                                    const int *slot, const long long *staging, Ctl *ctl, int mode,
                                                    int flags) {
    constexpr int NCH = THERM ? CH_ALL : CH_MOM_END;
    const double dt = ctl->dt;
    unsigned status = 0;
    double isc[NCH];
#pragma unroll
    for (int c = 0; c < NCH; ++c) isc[c] = ctl->inv_scale[c];
    // the fused G2P that follows takes its tiles from 0 (it starts after
    // this kernel ends, and the previous one has ended)
    if (blockIdx.x == 0 && threadIdx.x == 0) ctl->next_g2p = 0;
    const int nitems = tiles ? ctl->n_touched_tiles : (int)P.ntiles;
    for (int w = blockIdx.x; w < nitems; w += gridDim.x)
        nodes_tile<R, THERM, LEAN>(P, Nd, bc, tiles, slot, staging, isc, dt, mode, flags, w, status);
    if (status) atomicOr(&ctl->status, status);
}

// ---------------------------------------------------------------- K4 G2P
// Node access for the G2P particle update: a shared-memory node block or the
// dense global arrays.
template <class R>
struct SmemNodes {
    // [B3][NS]: per node v(3), dv(3) contiguous (FP32 padded to 8 words), so
    // one node is two 16-byte loads (FP32) or three (FP64)
    static constexpr int NS = (sizeof(R) == 4) ? 8 : 6;
    const R *nb;
    int B, B3;
    int org[3];   // node coordinate of block element 0
    __device__ __forceinline__ R get(int c, int i, int j, int k) const {
        return nb[(((k - org[2]) * B + (j - org[1])) * B + (i - org[0])) * NS + c];
    }
};
template <class R>
struct GlobalNodes {
    const R *v[3];
    const R *dv[3];
    Params P;
    __device__ __forceinline__ R get(int c, int i, int j, int k) const {
        long long n = node_index(P, i, j, k);
        if (n < 0) return R(0);
        return c < 3 ? v[c][n] : dv[c - 3][n];
    }
};

// Velocity interpolation weights of scheme `sch` along axis d, as
// bilin_interp_two / quadratic_interp_two / cubic_interp_two build them
// (interpolants.H:583-656, 863-1006, 1225-1366): scheme 1 is cell-relative
// linear on offsets 0,1; schemes 2/3 use that spline along every axis over
// the axis's compute_bounds range.
template <class R>
__device__ __forceinline__ void interp_axis(const SplineTables &t, const Params &P, int sch, int d, double x, int i,
                                            R w[4]) {
    int bmin, bmax;
    stencil_bounds(i, P.nc[d], P.order[d], P.periodic[d], bmin, bmax);
    for (int s = 0; s < 4; ++s) {
        const int l = s - 1;
        R val = R(0);
        if (sch == 1) {
            const double r = (x - (P.plo[d] + i * P.dx[d])) * P.dxi[d];
            val = (l == 0) ? (R)(1.0 - r) : (l == 1 ? (R)r : R(0));
        } else if (l >= bmin && l < bmax) {
            int ty = shape_type(i + l, P.nc[d], P.periodic[d]);
            const double r = (x - (P.plo[d] + (i + l) * P.dx[d])) * P.dxi[d];
            R der;
            spline_eval<R>(t, sch, ty, r, val, der);
        }
        w[s] = val;
    }
}

// interpolate_from_grid for one particle (mpm_particle_grid_ops.cpp:972-1096).
// FLIP blend, F update and strain rate from the interpolated velocity,
// velocity increment and velocity gradient (mpm_particle_grid_ops.cpp:1030-1094).
template <class R>
__device__ __forceinline__ void g2p_finish(const Params &P, bool upd_vel, bool upd_sr, const R vpic[3],
                                           const R dpic[3], const R gv[3][3], R v[3], R vp[3], R E[9], R sr[6],
                                           double dt, double &jfac) {
    jfac = 1.0;
    if (upd_vel) {
        const R a = (R)P.alpha;
        for (int d = 0; d < 3; ++d) {
            vp[d] = vpic[d];
            v[d] = a * v[d] + a * dpic[d] + (R(1) - a) * vpic[d];
        }
    }
    if (upd_sr && sizeof(R) == 8) {
        // FP64 state holds F itself: get_deformation_gradient_tensor
        // (interpolants.H:1732-1787), F <- (I + L dt) F, in the reference's
        // operation order with every product and sum rounded on its own (no
        // fused multiply-add), so F and J = det F follow the reference's
        // rounding step by step
        double nrm = 0.0;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) nrm = __dadd_rn(nrm, __dmul_rn((double)gv[a][b], (double)gv[a][b]));
        if (!(nrm >= 1.0e10)) {
            double L[3][3], Fo[3][3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    const double gd = __dmul_rn((double)gv[a][b], dt);
                    L[a][b] = (a == b) ? __dadd_rn(1.0, gd) : gd;
                    Fo[a][b] = (double)E[a * 3 + b];
                }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double acc = __dmul_rn(L[a][0], Fo[0][b]);
                    acc = __dadd_rn(acc, __dmul_rn(L[a][1], Fo[1][b]));
                    acc = __dadd_rn(acc, __dmul_rn(L[a][2], Fo[2][b]));
                    E[a * 3 + b] = (R)acc;
                }
        }
        int ind = 0;
        for (int d1 = 0; d1 < 3; ++d1)
            for (int d2 = d1; d2 < 3; ++d2) sr[ind++] = R(0.5) * (gv[d1][d2] + gv[d2][d1]);
    } else if (upd_sr) {
        // FP32 state holds E = F - I: the same update on F = I + E reads
        // E' = E + (L dt) + (L dt) E, which keeps small strains resolved
        R nrm = R(0);
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) nrm += gv[a][b] * gv[a][b];
        if (!(nrm >= R(1.0e10))) {
            R Ld[3][3], En[9];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) Ld[a][b] = gv[a][b] * (R)dt;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    R acc = E[a * 3 + b] + Ld[a][b];
                    for (int c = 0; c < 3; ++c) acc += Ld[a][c] * E[c * 3 + b];
                    En[a * 3 + b] = acc;
                }
            for (int q = 0; q < 9; ++q) E[q] = En[q];
            // det(I + L dt) in FP64: J = det F follows F' = (I + L dt) F
            // multiplicatively (kept in FP64 by the mixed-precision path)
            double a[3][3];
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) a[r][c] = (r == c ? 1.0 : 0.0) + (double)gv[r][c] * dt;
            jfac = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                   a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
        }
        int ind = 0;
        for (int d1 = 0; d1 < 3; ++d1)
            for (int d2 = d1; d2 < 3; ++d2) sr[ind++] = R(0.5) * (gv[d1][d2] + gv[d2][d1]);
    }
}

template <class R, int ORD, class NodeAcc>
__device__ __forceinline__ void g2p_particle_generic(const SplineTables &tab, const Params &P, const NodeAcc &na,
                                             const double x[3], const int iv[3], bool upd_vel, bool upd_sr, R v[3],
                                             R vp[3], R E[9], R sr[6], double dt, double &jfac) {
    // uniform quadratic: the 3-node window of the nearest-node bin (every
    // node with a non-zero weight), the same bin as the sort key's
    constexpr int W = (ORD == 2) ? 3 : Stc<ORD>::W, LO = Stc<ORD>::LO;
    AxisW<R, W> ax, ay, az;
    int base[3];
    if constexpr (ORD == 2) {
        AxisW<R, W> *a[3] = {&ax, &ay, &az};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int n0 = dual_bin(P, d, x[d]);
            dual_axis_weights<R>(tab, P, d, dual_x(P, d, x[d]), n0, false, *a[d]);
            base[d] = n0 - 1;
        }
    } else {
        axis_weights<R, W, LO>(tab, P, 0, x[0], iv[0], ax);
        axis_weights<R, W, LO>(tab, P, 1, x[1], iv[1], ay);
        axis_weights<R, W, LO>(tab, P, 2, x[2], iv[2], az);
#pragma unroll
        for (int d = 0; d < 3; ++d) base[d] = iv[d] + LO;
    }
    R vpic[3] = {R(0), R(0), R(0)}, dpic[3] = {R(0), R(0), R(0)};
    R gv[3][3] = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
    const bool generic = (ORD == 0);
#pragma unroll
    for (int sz = 0; sz < W; ++sz) {
#pragma unroll
        for (int sy = 0; sy < W; ++sy) {
#pragma unroll
            for (int sx = 0; sx < W; ++sx) {
                const R wx = ax.w[sx], wy = ay.w[sy], wz = az.w[sz];
                const R dx = ax.dw[sx], dy = ay.dw[sy], dz = az.dw[sz];
                if (wx == R(0) && dx == R(0)) continue;
                if (wy == R(0) && dy == R(0)) continue;
                if (wz == R(0) && dz == R(0)) continue;
                const int ni = base[0] + sx, nj = base[1] + sy, nk = base[2] + sz;
                const R nv[3] = {na.get(0, ni, nj, nk), na.get(1, ni, nj, nk), na.get(2, ni, nj, nk)};
                if (upd_vel && !generic) {
                    const R N = wx * wy * wz;
                    for (int d = 0; d < 3; ++d) {
                        vpic[d] += N * nv[d];
                        dpic[d] += N * na.get(3 + d, ni, nj, nk);
                    }
                }
                if (upd_sr) {
                    const R g[3] = {dx * wy * wz, wx * dy * wz, wx * wy * dz};
                    for (int d1 = 0; d1 < 3; ++d1)
                        for (int d2 = 0; d2 < 3; ++d2) gv[d1][d2] += nv[d1] * g[d2];
                }
            }
        }
    }
    if (upd_vel && generic) {
        // per-component scheme (order of the velocity component's axis)
        for (int dim = 0; dim < 3; ++dim) {
            const int sch = P.order[dim];
            R wx[4], wy[4], wz[4];
            interp_axis<R>(tab, P, sch, 0, x[0], iv[0], wx);
            interp_axis<R>(tab, P, sch, 1, x[1], iv[1], wy);
            interp_axis<R>(tab, P, sch, 2, x[2], iv[2], wz);
            for (int sz = 0; sz < 4; ++sz)
                for (int sy = 0; sy < 4; ++sy)
                    for (int sx = 0; sx < 4; ++sx) {
                        const R N = wx[sx] * wy[sy] * wz[sz];
                        if (N == R(0)) continue;
                        const int ni = iv[0] - 1 + sx, nj = iv[1] - 1 + sy, nk = iv[2] - 1 + sz;
                        vpic[dim] += N * na.get(dim, ni, nj, nk);
                        dpic[dim] += N * na.get(3 + dim, ni, nj, nk);
                    }
        }
    }
    g2p_finish<R>(P, upd_vel, upd_sr, vpic, dpic, gv, v, vp, E, sr, dt, jfac);
}

// Interpolation over a WN^3 window of the shared-memory node block
// (interpolate_from_grid, mpm_particle_grid_ops.cpp:972-1094), sum-factorized:
// along each x row  a = sum wx v,  b = sum dwx v,  c = sum wx dv;  over the
// rows of a z-slice  Sv = sum wy a,  Sy = sum dwy a,  Sx = sum wy b,
// Sd = sum wy c;  over the slices  v_pic = sum wz Sv,  dv_pic = sum wz Sd and
// grad v = (sum wz Sx, sum wz Sy, sum dwz Sv)  (the columns of
// sum v (x) grad N with grad N = (dwx wy wz, wx dwy wz, wx wy dwz)).  A node
// costs 5 FMAs (FP32: 4 packed and 1 scalar) instead of 15 plus the
// products N and grad N.
template <class R, int WN>
__device__ __forceinline__ void g2p_window(const SmemNodes<R> &na, const int base[3], const R wx[WN], const R dwx[WN],
                                           const R wy[WN], const R dwy[WN], const R wz[WN], const R dwz[WN],
                                           bool upd_vel, bool upd_sr, R vpic[3], R dpic[3], R gv[3][3]) {
    constexpr int NS = SmemNodes<R>::NS;
    const int B = na.B;
    const int i0 = ((base[2] - na.org[2]) * B + (base[1] - na.org[1])) * B + (base[0] - na.org[0]);
    const R *nb = na.nb;
    if constexpr (sizeof(R) == 4) {
        const float2 z2 = make_float2(0.f, 0.f);
        // slice-summed (x, y) pairs: v_pic (x, y), (v_pic z, dv_pic x),
        // dv_pic (y, z); gradient columns 0, 1, 2 for rows (x, y) and z
        float2 V01 = z2, V2D0 = z2, D12 = z2, G0 = z2, G1 = z2, G2 = z2;
        float g0z = 0.f, g1z = 0.f, g2z = 0.f;
#pragma unroll
        for (int sz = 0; sz < WN; ++sz) {
            float2 Sv01 = z2, Sv2d0 = z2, Sd12 = z2, Sy01 = z2, Sx01 = z2;
            float Sy2 = 0.f, Sx2 = 0.f;
#pragma unroll
            for (int sy = 0; sy < WN; ++sy) {
                const int row = i0 + (sz * B + sy) * B;
                float2 a01 = z2, a2c0 = z2, c12 = z2, b01 = z2;
                float b2 = 0.f;
#pragma unroll
                for (int sx = 0; sx < WN; ++sx) {
                    const float *q = nb + (row + sx) * NS;
                    const float4 va = *reinterpret_cast<const float4 *>(q);
                    const float2 wxx = make_float2(wx[sx], wx[sx]);
                    a01 = __ffma2_rn(wxx, make_float2(va.x, va.y), a01);
                    a2c0 = __ffma2_rn(wxx, make_float2(va.z, va.w), a2c0);
                    if (upd_vel) c12 = __ffma2_rn(wxx, *reinterpret_cast<const float2 *>(q + 4), c12);
                    if (upd_sr) {
                        b01 = __ffma2_rn(make_float2(dwx[sx], dwx[sx]), make_float2(va.x, va.y), b01);
                        b2 = fmaf(dwx[sx], va.z, b2);
                    }
                }
                const float2 wyy = make_float2(wy[sy], wy[sy]), dyy = make_float2(dwy[sy], dwy[sy]);
                Sv01 = __ffma2_rn(wyy, a01, Sv01);
                Sv2d0 = __ffma2_rn(wyy, a2c0, Sv2d0);
                if (upd_vel) Sd12 = __ffma2_rn(wyy, c12, Sd12);
                if (upd_sr) {
                    Sy01 = __ffma2_rn(dyy, a01, Sy01);
                    Sy2 = fmaf(dwy[sy], a2c0.x, Sy2);
                    Sx01 = __ffma2_rn(wyy, b01, Sx01);
                    Sx2 = fmaf(wy[sy], b2, Sx2);
                }
            }
            const float2 wzz = make_float2(wz[sz], wz[sz]), dzz = make_float2(dwz[sz], dwz[sz]);
            V01 = __ffma2_rn(wzz, Sv01, V01);
            V2D0 = __ffma2_rn(wzz, Sv2d0, V2D0);
            D12 = __ffma2_rn(wzz, Sd12, D12);
            if (upd_sr) {
                G0 = __ffma2_rn(wzz, Sx01, G0);
                g0z = fmaf(wz[sz], Sx2, g0z);
                G1 = __ffma2_rn(wzz, Sy01, G1);
                g1z = fmaf(wz[sz], Sy2, g1z);
                G2 = __ffma2_rn(dzz, Sv01, G2);
                g2z = fmaf(dwz[sz], Sv2d0.x, g2z);
            }
        }
        vpic[0] += V01.x;
        vpic[1] += V01.y;
        vpic[2] += V2D0.x;
        dpic[0] += V2D0.y;
        dpic[1] += D12.x;
        dpic[2] += D12.y;
        gv[0][0] += G0.x;
        gv[1][0] += G0.y;
        gv[2][0] += g0z;
        gv[0][1] += G1.x;
        gv[1][1] += G1.y;
        gv[2][1] += g1z;
        gv[0][2] += G2.x;
        gv[1][2] += G2.y;
        gv[2][2] += g2z;
    } else {
        R V[3] = {R(0), R(0), R(0)}, D[3] = {R(0), R(0), R(0)};
        R G[3][3] = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
#pragma unroll
        for (int sz = 0; sz < WN; ++sz) {
            R Sv[3] = {R(0), R(0), R(0)}, Sd[3] = {R(0), R(0), R(0)}, Sy[3] = {R(0), R(0), R(0)},
              Sx[3] = {R(0), R(0), R(0)};
#pragma unroll
            for (int sy = 0; sy < WN; ++sy) {
                const int row = i0 + (sz * B + sy) * B;
                R a[3] = {R(0), R(0), R(0)}, bx[3] = {R(0), R(0), R(0)}, c[3] = {R(0), R(0), R(0)};
#pragma unroll
                for (int sx = 0; sx < WN; ++sx) {
                    const R *q = nb + (row + sx) * NS;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        a[d] = fma(wx[sx], q[d], a[d]);
                        if (upd_vel) c[d] = fma(wx[sx], q[3 + d], c[d]);
                        if (upd_sr) bx[d] = fma(dwx[sx], q[d], bx[d]);
                    }
                }
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    Sv[d] = fma(wy[sy], a[d], Sv[d]);
                    if (upd_vel) Sd[d] = fma(wy[sy], c[d], Sd[d]);
                    if (upd_sr) {
                        Sy[d] = fma(dwy[sy], a[d], Sy[d]);
                        Sx[d] = fma(wy[sy], bx[d], Sx[d]);
                    }
                }
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                V[d] = fma(wz[sz], Sv[d], V[d]);
                D[d] = fma(wz[sz], Sd[d], D[d]);
                if (upd_sr) {
                    G[d][0] = fma(wz[sz], Sx[d], G[d][0]);
                    G[d][1] = fma(wz[sz], Sy[d], G[d][1]);
                    G[d][2] = fma(dwz[sz], Sv[d], G[d][2]);
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            vpic[d] += V[d];
            dpic[d] += D[d];
#pragma unroll
            for (int j = 0; j < 3; ++j) gv[d][j] += G[d][j];
        }
    }
}

// G2P of one particle from the shared-memory node block: the interior fast
// path (fixed spline pieces; quadratic on its 3-node window) when every
// stencil node of the particle's cell has the interior shape type, else the
// table-driven path.
template <class R, int ORD>
__device__ __forceinline__ void g2p_particle_smem(const SplineTables &tab, const Params &P, const SmemNodes<R> &na,
                                                  const double x[3], const int iv[3], bool upd_vel, bool upd_sr,
                                                  R v[3], R vp[3], R E[9], R sr[6], double dt, double &jfac) {
    R vpic[3] = {R(0), R(0), R(0)}, dpic[3] = {R(0), R(0), R(0)};
    R gv[3][3] = {{R(0), R(0), R(0)}, {R(0), R(0), R(0)}, {R(0), R(0), R(0)}};
    if constexpr (ORD == 2) {
        // the window of the particle's nearest-node bin (the bin its tile
        // was sorted by), fixed pieces on interior axes
        AxisW<R, 3> a[3];
        int base[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int n0 = dual_bin(P, d, x[d]);
            const bool in = P.periodic[d] || (n0 >= 3 && n0 <= P.nc[d] - 3);
            const double xw = dual_x(P, d, x[d]);
            if (in)
                interior_weights<R, 2>((R)((xw - (P.plo[d] + n0 * P.dx[d])) * P.dxi[d]), (R)P.dxi[d], a[d]);
            else
                dual_axis_weights<R>(tab, P, d, xw, n0, false, a[d]);
            base[d] = n0 - 1;
        }
        g2p_window<R, 3>(na, base, a[0].w, a[0].dw, a[1].w, a[1].dw, a[2].w, a[2].dw, upd_vel, upd_sr, vpic, dpic,
                         gv);
        g2p_finish<R>(P, upd_vel, upd_sr, vpic, dpic, gv, v, vp, E, sr, dt, jfac);
        return;
    }
    if constexpr (ORD == 3) {
        // cubic: the 4x4x4 window of the particle's cell; fixed spline pieces
        // on interior axes, the boundary-aware tables (zero outside
        // compute_bounds) elsewhere; nodes outside the domain are 0 in the block
        AxisW<R, 4> a[3];
        int base[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const bool in = P.periodic[d] || (iv[d] >= 3 && iv[d] <= P.nc[d] - 4);
            if (in)
                interior_weights<R, 3>((R)((x[d] - (P.plo[d] + iv[d] * P.dx[d])) * P.dxi[d]), (R)P.dxi[d], a[d]);
            else
                axis_weights<R, 4, -1>(tab, P, d, x[d], iv[d], a[d]);
            base[d] = iv[d] - 1;
        }
        g2p_window<R, 4>(na, base, a[0].w, a[0].dw, a[1].w, a[1].dw, a[2].w, a[2].dw, upd_vel, upd_sr, vpic, dpic,
                         gv);
        g2p_finish<R>(P, upd_vel, upd_sr, vpic, dpic, gv, v, vp, E, sr, dt, jfac);
        return;
    }
    bool inter = (ORD != 0);
#pragma unroll
    for (int d = 0; d < 3; ++d)
        inter = inter && ((ORD == 1) || P.periodic[d] || (iv[d] >= 3 && iv[d] <= P.nc[d] - 4));
    if (!inter) {
        g2p_particle_generic<R, ORD>(tab, P, na, x, iv, upd_vel, upd_sr, v, vp, E, sr, dt, jfac);
        return;
    }
    if (ORD == 1 || ORD == 3) {
        constexpr int WN = (ORD == 1) ? 2 : 4;
        constexpr int OW = (ORD == 0) ? 3 : ORD;  // keeps the template argument valid when ORD == 0
        AxisW<R, WN> a[3];
        int base[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            axis_weights_interior<R, OW>(P, d, x[d], iv[d], a[d]);
            base[d] = iv[d] + Stc<OW>::LO;
        }
        g2p_window<R, WN>(na, base, a[0].w, a[0].dw, a[1].w, a[1].dw, a[2].w, a[2].dw, upd_vel, upd_sr, vpic, dpic,
                          gv);
    }
    g2p_finish<R>(P, upd_vel, upd_sr, vpic, dpic, gv, v, vp, E, sr, dt, jfac);
}

// G2P of one particle through any node accessor (the unfused L5 path).
template <class R, int ORD, class NodeAcc>
__device__ __forceinline__ void g2p_particle(const SplineTables &tab, const Params &P, const NodeAcc &na,
                                             const double x[3], const int iv[3], bool upd_vel, bool upd_sr, R v[3],
                                             R vp[3], R E[9], R sr[6], double dt, double &jfac) {
    g2p_particle_generic<R, ORD>(tab, P, na, x, iv, upd_vel, upd_sr, v, vp, E, sr, dt, jfac);
}


// moveParticles for one particle (mpm_particle_timestep.cpp:326-576).
// LEAN: no level-set bodies and no UDF walls (compiled out)
template <class R, bool LEAN = false>
__device__ __forceinline__ void move_particle(const Params &P, const NodeBCArgs &bc, int phase, double x[3], R v[3],
                                              const R vp[3], double dt, unsigned &status) {
    for (int d = 0; d < 3; ++d) x[d] += (double)vp[d] * dt;
    double rin[3] = {(double)v[0], (double)v[1], (double)v[2]};
    double rout[3] = {rin[0], rin[1], rin[2]};
    if (!LEAN && P.num_bodies > 0 && phase == 0) {
        int hit = -1;
        double minphi = kTiny;
        for (int b = 0; b < P.num_bodies; ++b) {
            if (!bc.ls[b]) continue;
            double ph, gg[3];
            ls_sample(P, bc.ls[b], x, ph, gg);
            if (ph < minphi) {
                minphi = ph;
                hit = b;
            }
        }
        if (hit >= 0) {
            double ph, nd[3];
            ls_sample(P, bc.ls[hit], x, ph, nd);
            double gm = sqrt(nd[0] * nd[0] + nd[1] * nd[1] + nd[2] * nd[2]);
            for (int d = 0; d < 3; ++d) nd[d] /= (gm + kTiny);
            int mp = applybc<double>(rin, rout, P.body[hit].wall_mu, nd, P.body[hit].mom_bc);
            if (mp < 0) status |= ST_BC;
            if (mp > 0)
                for (int d = 0; d < 3; ++d) x[d] += 2.0 * fabs(minphi) * nd[d];
            for (int d = 0; d < 3; ++d) v[d] = (R)rout[d];
        }
    }
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
        const bool lo = x[dir] < P.plo[dir];
        const bool hi = !lo && x[dir] > P.phi[dir];
        if (!lo && !hi) continue;
        double wv[3];
        for (int d = 0; d < 3; ++d) wv[d] = lo ? P.wvel_lo[dir * 3 + d] : P.wvel_hi[dir * 3 + d];
        const double *tab = LEAN ? nullptr : bc.udf[hi ? 1 : 0][dir];
        if (tab) {
            const int p0 = (dir == 0) ? 1 : 0, p1 = (dir == 2) ? 1 : 2;
            double f0 = (x[p0] - P.plo[p0]) / P.dx[p0], f1 = (x[p1] - P.plo[p1]) / P.dx[p1];
            f0 = fmax(0.0, fmin((double)P.nc[p0], f0));
            f1 = fmax(0.0, fmin((double)P.nc[p1], f1));
            int j0 = (int)f0, j1 = min(j0 + 1, P.nc[p0]);
            int k0 = (int)f1, k1 = min(k0 + 1, P.nc[p1]);
            double wx1 = f0 - j0, wx0 = 1.0 - wx1, wy1 = f1 - k0, wy0 = 1.0 - wy1;
            int n1 = P.nc[p1] + 1;
            for (int c = 0; c < 3; ++c)
                wv[c] = wx0 * wy0 * tab[(j0 * n1 + k0) * 3 + c] + wx0 * wy1 * tab[(j0 * n1 + k1) * 3 + c] +
                        wx1 * wy0 * tab[(j1 * n1 + k0) * 3 + c] + wx1 * wy1 * tab[(j1 * n1 + k1) * 3 + c];
        }
        for (int d = 0; d < 3; ++d) rin[d] -= wv[d];
        double nd[3] = {0, 0, 0};
        nd[dir] = lo ? 1.0 : -1.0;
        int mp = applybc<double>(rin, rout, lo ? P.wmu_lo[dir] : P.wmu_hi[dir], nd, lo ? P.bclo[dir] : P.bchi[dir]);
        if (mp < 0) status |= ST_BC;
        if (mp > 0) x[dir] = lo ? 2.0 * P.plo[dir] - x[dir] : 2.0 * P.phi[dir] - x[dir];
        for (int c = 0; c < 3; ++c) v[c] = (R)(rout[c] + wv[c]);
    }
}

// updateVolume + apply_constitutive_model for one phase-0 particle
// (mpm_particle_timestep.cpp:131-182, mpm_particle_container.cpp:43-142).
// J, the Tait pressure and the density division are FP64.
// (1/J)^gamma of the Tait EOS: a whole-number gamma (7 for water) by
// repeated squaring, a few ulp from pow at a small part of its cost
__device__ __forceinline__ double tait_power(double x, const Material &mt) {
    int n = mt.ipow;
    if (n == 0) return pow(x, mt.gamma);
    double r = 1.0, b = x;
    while (n) {
        if (n & 1) r *= b;
        b *= b;
        n >>= 1;
    }
    return r;
}

// LEAN: total strain, linear-elastic and Tait materials only (the others
// compiled out)
template <class R, bool LEAN = false>
__device__ __forceinline__ void volume_stress(const Params &P, const Material &mt, const R E[9], R vol0, R mass,
                                              const R sr[6], R eps[6], R sig[6], R &vol, R &rho, double &J, R &pres,
                                              double dt, double asr, bool do_volume, bool do_stress) {
    double e[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) e[q] = (double)E[q];
    // J = det F in FP64: with FP64 state E holds F and det F is formed in
    // the reference's order (updateVolume, mpm_particle_timestep.cpp:160-163)
    // without fused multiply-adds; with FP32 state (E = F - I) the caller's
    // J, which follows F multiplicatively in FP64 (det(I + L dt) per F
    // update), since det of the FP32 F would carry its rounding
    const double det = (sizeof(R) == 8) ? det_ref(e) : J;
    if (do_volume) {
        const double V = (double)vol0 * det;
        J = det;
        vol = (R)V;
        rho = (R)((double)mass / V);
    }
    if (do_stress) {
        // one rounding, written out: left to the compiler, the contraction of
        // this product could differ between the kernel variants that inline
        // it (lean or full G2P, single-scene or batched)
#pragma unroll
        for (int d = 0; d < 6; ++d) eps[d] = fma((R)dt, sr[d], eps[d]);
        eps[0] += (R)(dt * asr);
        eps[3] += (R)(dt * asr);
        eps[5] += (R)(dt * asr);
        if (!LEAN && P.delta_strain) {
            // apply_constitutive_model_delta (mpm_particle_container.cpp:178-272):
            // sigma += C : (dt D + applied strain-rate increment), linear elastic
            if (mt.model == 0) {
                R de[6], ds[6];
#pragma unroll
                for (int d = 0; d < 6; ++d) de[d] = (R)dt * sr[d];
                de[0] += (R)(dt * asr);
                de[3] += (R)(dt * asr);
                de[5] += (R)(dt * asr);
                linear_elastic<R>(de, ds, (R)mt.E, (R)mt.nu);
#pragma unroll
                for (int d = 0; d < 6; ++d) sig[d] += ds[d];
            }
        } else if (mt.model == 0) {
            linear_elastic<R>(eps, sig, (R)mt.E, (R)mt.nu);
        } else if (LEAN || mt.model == 1) {
            // Tait EOS p = K ((1/J)^gamma - 1) (mpm_particle_container.cpp:113-120), FP64
            const double pj = mt.K * (tait_power(1.0 / det, mt) - 1.0);
            pres = (R)pj;
            newtonian<R>(sr, sig, (R)mt.mu, (R)pj);
        } else {
            // neo-Hookean (constitutive_models.H:161-250), FP64, J = max(det F,
            // 1e-12): b - I from F itself (FP64 state, b = F F^T as the
            // reference forms it) or from E = F - I (FP32 state: b - I =
            // E + E^T + E E^T keeps small strains resolved)
            const double mu = mt.E / (2.0 * (1.0 + mt.nu));
            const double lambda = mt.E * mt.nu / ((1.0 + mt.nu) * (1.0 - 2.0 * mt.nu));
            const double Jc = fmax(det, 1.e-12);
            const double vol = lambda * log(Jc) / Jc, muJ = mu / Jc;
            auto bm = [&](int i, int j) {
                if (sizeof(R) == 8)
                    return (e[3 * i] * e[3 * j] + e[3 * i + 1] * e[3 * j + 1] + e[3 * i + 2] * e[3 * j + 2]) -
                           (i == j ? 1.0 : 0.0);
                return e[3 * i + j] + e[3 * j + i] +
                       (e[3 * i] * e[3 * j] + e[3 * i + 1] * e[3 * j + 1] + e[3 * i + 2] * e[3 * j + 2]);
            };
            sig[0] = (R)(muJ * bm(0, 0) + vol);
            sig[1] = (R)(muJ * bm(0, 1));
            sig[2] = (R)(muJ * bm(0, 2));
            sig[3] = (R)(muJ * bm(1, 1) + vol);
            sig[4] = (R)(muJ * bm(1, 2));
            sig[5] = (R)(muJ * bm(2, 2) + vol);
        }
    }
}

template <class R>
__device__ __forceinline__ bool all_finite(const R *a, int n) {
    bool ok = true;
    for (int i = 0; i < n; ++i) ok = ok && isfinite((double)a[i]);
    return ok;
}

// Fused K4: one CTA per non-empty tile.  The tile's node block (velocity
// and delta-velocity, halo included) is staged in shared memory once; each
// particle of the tile is gathered from storage A through the sort
// permutation and written to storage B at its sorted position, so the
// particle arrays are physically re-ordered by cell every step at no extra
// pass.  GM_VEL updates velocity in place in A instead.
// L2 prefetch of the fields the fused G2P reads for storage index i.  The
// storage is in the previous step's sorted order, and particles rarely change
// bins in one step, so storage index k holds (nearly always) the particle of
// sorted position k: prefetching index k + 2 blockDim.x (two iterations
// ahead; measured against one and three ahead and none) overlaps later
// iterations' loads with this one's arithmetic.
#ifndef EXG_G2P_PREFETCH
#define EXG_G2P_PREFETCH 2
#endif
template <class R>
__device__ __forceinline__ void prefetch_particle(const Parts<R> &A, long long i, bool with_vp) {
    auto pf = [](const void *q) { asm volatile("prefetch.global.L2 [%0];" ::"l"(q)); };
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        pf(A.x[d] + i);
        pf(A.v[d] + i);
        if (with_vp) pf(A.vp[d] + i);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) pf(A.E[q] + i);
#pragma unroll
    for (int c = 0; c < 6; ++c) pf(A.eps[c] + i);
    pf(A.pres + i);
    pf(A.mass + i);
    pf(A.vol0 + i);
    pf(A.mat + i);
    pf(A.phase + i);
    pf(A.pid + i);
}

// One tile of the fused G2P: stage the tile's node block (v, dv and halo)
// in shared memory, then update each of the tile's particles.
template <class R, int ORD, bool LEAN>
__device__ __forceinline__ void g2p_tile(const SplineTables *tab, R *nb, const Params &P, const Parts<R> &A,
                                         const Parts<R> &Bo, const Nodes<R> &Nd, const NodeBCArgs &bc,
                                         const Material *mats, const int *active, const int *start, const int *count,
                                         const int32_t *perm, int mode, int w, double dt, double asr, bool upd_vel,
                                         float (&run_b)[CH_ALL], double &run_speed, bool &red, unsigned &status,
                                         bool staged = false, int kbeg = 0, int kend = 1 << 30,
                                         long long np_cap = 1ll << 62) {
    const int B = P.B, B3 = B * B * B;
    const int t = active[w];
    int tc[3];
    tile_coords(P, t, tc);
    SmemNodes<R> na;
    na.nb = nb;
    na.B = B;
    na.B3 = B3;
    for (int d = 0; d < 3; ++d) na.org[d] = tc[d] * P.T - P.hlo;
    if (!staged) {
        // the node block by plain loads (the caller did not stage it by TMA)
        for (int idx = threadIdx.x; idx < B3; idx += blockDim.x) {
            const int bx = idx % B, by = (idx / B) % B, bz = idx / (B * B);
            const long long ni = node_index(P, na.org[0] + bx, na.org[1] + by, na.org[2] + bz);
            R *q = nb + idx * SmemNodes<R>::NS;
            for (int c = 0; c < 3; ++c) {
                q[c] = ni >= 0 ? Nd.c[EXG_N_VEL + c][ni] : R(0);
                q[3 + c] = ni >= 0 ? Nd.c[EXG_N_DVEL + c][ni] : R(0);
            }
        }
        __syncthreads();
    }
    const int s0 = start[t], n = count[t];
    // a velocity update overwrites v' of every phase-0 particle: the stored
    // v' is read only for rigid particles and for G2P without it
    const bool vel_only = mode == GM_VEL, fresh_vp = vel_only || upd_vel;
    // the particles kbeg .. kend - 1 of the tile (one work item)
    int k_end = s0 + min(n, kend);
    if (kbeg < 0 || kbeg >= n || s0 < 0 || (long long)s0 + n > np_cap) {
        status |= ST_BOUNDS;
        k_end = 0;
    }
    for (int k = s0 + kbeg + threadIdx.x; k < k_end; k += blockDim.x) {
        if (EXG_G2P_PREFETCH && k + EXG_G2P_PREFETCH * (int)blockDim.x < s0 + n)
            prefetch_particle<R>(A, k + EXG_G2P_PREFETCH * blockDim.x, !fresh_vp);
        const int p = perm[k];
        if (p < 0 || (long long)p >= np_cap) {
            status |= ST_BOUNDS;
            continue;
        }
        const int phase = A.phase[p];
        double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
        const bool read_vp = !vel_only && (phase != 0 || !upd_vel);
        R v[3], vp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = A.v[d][p];
            vp[d] = read_vp ? A.vp[d][p] : R(0);
        }
        if (vel_only) {
            if (phase == 0) {
                int iv[3];
                cell_of(P, x, iv);
                R E[9], sr[6];
                double jf;
                g2p_particle_smem<R, ORD>(*tab, P, na, x, iv, true, false, v, vp, E, sr, dt, jf);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    A.v[d][p] = v[d];
                    A.vp[d][p] = vp[d];
                }
            }
            continue;
        }
        R E[9], sr[6], eps[6], sig[6];
        R vol, rho, pres;
        double J = A.J[p], jf = 1.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) E[q] = A.E[q][p];
#pragma unroll
        for (int c = 0; c < 6; ++c) eps[c] = A.eps[c][p];
        pres = A.pres[p];
        if (phase != 0) {
            // rigid particles are only advected: keep their stored fields
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                sr[c] = A.sr[c][p];
                sig[c] = A.sig[c][p];
            }
            vol = A.vol[p];
            rho = A.rho[p];
        } else if (!LEAN && P.delta_strain) {
            // the incremental formulation adds to the stored stress
#pragma unroll
            for (int c = 0; c < 6; ++c) sig[c] = A.sig[c][p];
        }
        const R mass = A.mass[p], vol0 = A.vol0[p];
        const int mi = A.mat[p];
        if (phase == 0) {
            int iv[3];
            cell_of(P, x, iv);
            g2p_particle_smem<R, ORD>(*tab, P, na, x, iv, upd_vel, true, v, vp, E, sr, dt, jf);
        }
        move_particle<R, LEAN>(P, bc, phase, x, v, vp, dt, status);
        // Redistribute's periodic wrap
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (P.periodic[d]) {
                const double L = P.phi[d] - P.plo[d];
                if (x[d] >= P.phi[d])
                    x[d] -= L;
                else if (x[d] < P.plo[d])
                    x[d] += L;
            }
        const Material mt = mats[mi];
        if (phase == 0) {
            J *= jf;  // FP32 state: J follows F multiplicatively in FP64
            volume_stress<R, LEAN>(P, mt, E, vol0, mass, sr, eps, sig, vol, rho, J, pres, dt, asr, true, true);
            if (!all_finite(v, 3) || !all_finite(sig, 6) || !isfinite((double)J)) status |= ST_NAN;
            // reductions for the next step (running per thread)
            int iv2[3];
            cell_of(P, x, iv2);
            const bool in = iv2[0] >= 0 && iv2[0] < P.nc[0] && iv2[1] >= 0 && iv2[1] < P.nc[1] && iv2[2] >= 0 &&
                            iv2[2] < P.nc[2];
            if (in) {
                const double vd[3] = {(double)v[0], (double)v[1], (double)v[2]};
                const float fv[3] = {(float)v[0], (float)v[1], (float)v[2]};
                float fsig[6];
#pragma unroll
                for (int c = 0; c < 6; ++c) fsig[c] = (float)sig[c];
                // FP32 state without temperature: the same FP32 bounds in
                // every G2P kernel (lean, full and batched), so a scene's
                // steps do not depend on which one runs it
                if (sizeof(R) == 4 && (LEAN || !P.use_temp)) {
                    lean_bounds_f(P, mt, (float)mass, fv, (float)vol, fsig, (float)rho, run_b, run_speed);
                } else {
                    double sd[6];
#pragma unroll
                    for (int c = 0; c < 6; ++c) sd[c] = (double)sig[c];
                    double q[3] = {0, 0, 0}, cp = 0, T = 0, kc = 0, Q = 0;
                    if (!LEAN && P.use_temp) {
                        for (int d = 0; d < 3; ++d) q[d] = (double)A.q[d][p];
                        cp = A.cp[p];
                        T = A.T[p];
                        kc = A.kc[p];
                        Q = A.Q[p];
                    }
                    double bnd[CH_ALL], speed;
                    particle_bounds<R>(P, mt, (double)mass, vd, (double)vol, sd, (double)rho, cp, T, kc, q, Q, bnd,
                                       speed);
#pragma unroll
                    for (int c = 0; c < CH_ALL; ++c) run_b[c] = fmaxf(run_b[c], __double2float_ru(bnd[c]));
                    run_speed = fmax(run_speed, speed);
                }
                red = true;
            }
        }
        // write B at the sorted position k
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            Bo.x[d][k] = x[d];
            Bo.v[d][k] = v[d];
            Bo.vp[d][k] = vp[d];
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            Bo.sr[c][k] = sr[c];
            Bo.eps[c][k] = eps[c];
            Bo.sig[c][k] = sig[c];
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) Bo.E[q][k] = E[q];
        Bo.vol[k] = vol;
        Bo.rho[k] = rho;
        Bo.J[k] = J;
        Bo.pres[k] = pres;
        Bo.mass[k] = mass;
        Bo.vol0[k] = vol0;
        Bo.mat[k] = mi;
        Bo.phase[k] = (uint8_t)phase;
        Bo.pid[k] = A.pid[p];
        if (!LEAN && P.use_temp) {
            Bo.T[k] = A.T[p];
            Bo.cp[k] = A.cp[p];
            Bo.kc[k] = A.kc[p];
            Bo.Q[k] = A.Q[p];
            for (int d = 0; d < 3; ++d) Bo.q[d][k] = A.q[d][p];
        }
    }
    __syncthreads();
}

// Launch variants of the fused G2P (threads per block, minimum resident
// blocks per SM); variant 0 is the default, the autotuner measures the
// others on the lean quadratic and cubic kernels.  Each particle's update is
// independent of the launch shape, so all variants give identical results.
constexpr int kG2PVariants = 3;
static_assert(kG2PVariants == EXG_NUM_VARIANTS, "the launchers dispatch EXG_NUM_VARIANTS G2P variants");
// threads per block, minimum blocks per SM:
//   FP32: (256, 2)  (192, 2)  (384, 1);   FP64: (256, 2)  (256, 1)  (384, 1)
// (192, 2) keeps 12 warps per SM, as (384, 1), with 170 registers a thread
// and two blocks whose barriers and node-block waits overlap.
template <class R, int V>
struct G2PVar {
    static constexpr int THREADS = (V == 0) ? EXG_G2P_THREADS : (V == 1 ? (sizeof(R) == 4 ? 192 : 256) : 384);
    static constexpr int MINB = (V == 0) ? EXG_G2P_MINB : (V == 1 ? (sizeof(R) == 4 ? 2 : 1) : 1);
};

// ---- TMA staging of the G2P node block (cp.async.bulk.tensor + mbarrier)
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Arms the barrier's current phase for `bytes` of transfer (one arrival).
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// One 4-D tensor box (node-record words, x, y, z) into shared memory,
// completing on the barrier.  Coordinates outside the tensor read zeros.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            unsigned long long *bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for a barrier phase: gives up after kTmaWaitLimit polls (each
// poll may itself suspend the warp for a while), so a transfer that never
// completes ends the kernel with ST_TIMEOUT instead of hanging it.
constexpr long long kTmaWaitLimit = 1ll << 24;
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity) {
    for (long long it = 0; it < kTmaWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// The active tile of fused-G2P work item `item`: the last w with
// item_start[w] <= item (every active tile has at least one item, so the
// starts increase strictly).
__device__ __forceinline__ int item_tile(const int *item_start, int nact, int item) {
    int lo = 0, hi = nact - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (item_start[mid] <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <class R, int ORD, bool LEAN, int V = 0>
__global__ void __launch_bounds__(G2PVar<R, V>::THREADS, G2PVar<R, V>::MINB) k_g2p_fused(Params P, Parts<R> A, Parts<R> Bo, Nodes<R> Nd, NodeBCArgs bc,
                                                        const Material *mats, const int *active, const int *start,
                                                        const int *count, const int32_t *perm,
                                                        const int *item_start, Ctl *ctl, int mode,
                                                        const __grid_constant__ CUtensorMap tmap, int use_tma,
                                                        long long np) {
    extern __shared__ __align__(128) unsigned char smraw[];
    SplineTables *tab = reinterpret_cast<SplineTables *>(smraw);
    const size_t tab_bytes = (sizeof(SplineTables) + 127) & ~size_t(127);
    // The dynamic shared memory follows the kernel's static shared variables
    // and is only 16-byte aligned, while a TMA tensor copy writes to a
    // 128-byte aligned shared address: the node blocks start at the next
    // 128-byte boundary after the tables (the launch adds 128 bytes for it).
    const unsigned nb_sa = smem_addr(smraw + tab_bytes);
    R *nb = reinterpret_cast<R *>(smraw + tab_bytes + ((128u - (nb_sa & 127u)) & 127u));
    load_tables(tab);
    const double dt = ctl->dt, time = ctl->time;
    const double asr = (time < P.applied_sr_time) ? P.applied_sr : 0.0;
    unsigned status = 0;
    if (use_tma && (smem_addr(nb) & 127u) != 0u) {
        // never taken with the padding above; checked before any copy is issued
        status |= ST_ALIGN;
        use_tma = 0;
    }
    const bool upd_vel = (mode != GM_STRAIN);
    // running per-thread maxima of the P2G bounds (float is enough for a
    // power-of-two scale with a factor-2 margin; rounded up on conversion)
    float run_b[CH_ALL];
#pragma unroll
    for (int c = 0; c < CH_ALL; ++c) run_b[c] = 0.0f;
    double run_speed = 0.0;  // largest CFL wave speed of the thread's particles
    bool red = false;
    // work items (chunks of kG2PChunk particles of a tile) are taken in turn
    // from a device counter (reset by k_nodes)
    const int nitems = ctl->n_g2p_items, nact = ctl->n_active_tiles;
    if (!use_tma) {
        __shared__ int s_item, s_w;
        for (;;) {
            if (threadIdx.x == 0) {
                s_item = atomicAdd(&ctl->next_g2p, 1);
                if (s_item < nitems) s_w = item_tile(item_start, nact, s_item);
            }
            __syncthreads();
            const int it = s_item;
            if (it >= nitems) break;
            const int w = s_w;
            int kb = (w >= 0 && w < nact) ? (it - item_start[w]) * kG2PChunk : -1;
            if (kb < 0) status |= ST_BOUNDS;
            g2p_tile<R, ORD, LEAN>(tab, nb, P, A, Bo, Nd, bc, mats, active, start, count, perm, mode, w, dt, asr,
                                   upd_vel, run_b, run_speed, red, status, false, kb, kb + kG2PChunk, np);
        }
    } else {
        // The node block of each tile comes by one TMA box from the nodal
        // kernel's interleaved records.  FP32: two buffers, the next tile's
        // block loads while this tile's particles are updated; FP64 (larger
        // blocks): one buffer, loaded between tiles.
        constexpr int NBUF = sizeof(R) == 4 ? 2 : 1;
        const int B = P.B;
        const size_t buf_words = (((size_t)B * B * B * SmemNodes<R>::NS * sizeof(R) + 127) & ~size_t(127)) / sizeof(R);
        const unsigned box_bytes = (unsigned)((size_t)B * B * B * SmemNodes<R>::NS * sizeof(R));
        __shared__ __align__(8) unsigned long long mbar[2];
        __shared__ int s_items[2], s_ws[2];
        auto issue = [&](int item, int b) {
            const int w = item_tile(item_start, nact, item);
            s_ws[b] = w;
            int tc[3];
            tile_coords(P, active[w], tc);
            mbar_expect_tx(&mbar[b], box_bytes);
            tma_load_4d(nb + b * buf_words, &tmap, 0, tc[0] * P.T - P.hlo, tc[1] * P.T - P.hlo, tc[2] * P.T - P.hlo,
                        &mbar[b]);
        };
        if (threadIdx.x == 0) {
            mbar_init(&mbar[0], 1);
            mbar_init(&mbar[1], 1);
            mbar_init_fence();
            const int i = atomicAdd(&ctl->next_g2p, 1);
            s_items[0] = i;
            if (i < nitems) issue(i, 0);
        }
        __syncthreads();
        unsigned ph[2] = {0u, 0u};
        int cur = 0;
        for (;;) {
            const int it = s_items[cur];
            if (it >= nitems) break;
            const int w = s_ws[cur];
            int kb = (w >= 0 && w < nact) ? (it - item_start[w]) * kG2PChunk : -1;
            if (kb < 0) status |= ST_BOUNDS;
            if (NBUF == 2 && threadIdx.x == 0) {
                // the other buffer's last tile is done (the block synchronised)
                const int i = atomicAdd(&ctl->next_g2p, 1);
                s_items[cur ^ 1] = i;
                if (i < nitems) issue(i, cur ^ 1);
            }
            const bool ok = mbar_wait(&mbar[cur], ph[cur]);
            ph[cur] ^= 1u;
            if (__syncthreads_or(!ok)) {
                // a transfer did not complete: flag it, and before leaving
                // wait (bounded) for the other buffer's transfer in flight
                status |= ST_TIMEOUT;
                if (NBUF == 2 && s_items[cur ^ 1] < nitems) mbar_wait(&mbar[cur ^ 1], ph[cur ^ 1]);
                break;
            }
            g2p_tile<R, ORD, LEAN>(tab, nb + cur * buf_words, P, A, Bo, Nd, bc, mats, active, start, count, perm,
                                   mode, w, dt, asr, upd_vel, run_b, run_speed, red, status, true, kb,
                                   kb + kG2PChunk, np);
            if (NBUF == 2) {
                cur ^= 1;
            } else {
                if (threadIdx.x == 0) {
                    const int i = atomicAdd(&ctl->next_g2p, 1);
                    s_items[0] = i;
                    if (i < nitems) issue(i, 0);
                }
                __syncthreads();
            }
        }
    }
    if (mode != GM_VEL) {
        double rb[CH_ALL];
#pragma unroll
        for (int c = 0; c < CH_ALL; ++c) rb[c] = (double)run_b[c];
        block_reduce_push(&ctl->bound_bits[0], &ctl->dtmin_bits, rb, P.dxmin / run_speed, red);
    }
    if (status) atomicOr(&ctl->status, status);
}

// Particles outside the domain belong to no tile, so the fused G2P does not
// write them; they follow the sorted ones in the re-ordered storage
// (removed particles stay in storage, inert, as AMReX-invalidated ones do).
template <class R>
__device__ __forceinline__ void copy_particle(const Parts<R> &A, long long i, Parts<R> &Bo, long long j, bool temp) {
    for (int d = 0; d < 3; ++d) {
        Bo.x[d][j] = A.x[d][i];
        Bo.v[d][j] = A.v[d][i];
        Bo.vp[d][j] = A.vp[d][i];
    }
    for (int c = 0; c < 6; ++c) {
        Bo.sr[c][j] = A.sr[c][i];
        Bo.eps[c][j] = A.eps[c][i];
        Bo.sig[c][j] = A.sig[c][i];
    }
    for (int q = 0; q < 9; ++q) Bo.E[q][j] = A.E[q][i];
    Bo.vol[j] = A.vol[i];
    Bo.mass[j] = A.mass[i];
    Bo.rho[j] = A.rho[i];
    Bo.J[j] = A.J[i];
    Bo.pres[j] = A.pres[i];
    Bo.vol0[j] = A.vol0[i];
    Bo.mat[j] = A.mat[i];
    Bo.phase[j] = A.phase[i];
    Bo.pid[j] = A.pid[i];
    if (temp) {
        Bo.T[j] = A.T[i];
        Bo.cp[j] = A.cp[i];
        Bo.kc[j] = A.kc[i];
        Bo.Q[j] = A.Q[i];
        for (int d = 0; d < 3; ++d) Bo.q[d][j] = A.q[d][i];
    }
}

template <class R>
__global__ void k_copy_lost(Parts<R> A, Parts<R> Bo, const uint32_t *key, long long np, Ctl *ctl, int temp) {
    if (ctl->lost == 0) return;  // the usual case: nothing to copy, no key to read
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= np || key[i] != 0xFFFFFFFFu) return;
    long long j = ctl->n_sorted + (long long)atomicAdd(&ctl->lost_fill, 1ull);
    copy_particle<R>(A, i, Bo, j, temp != 0);
}

// ---------------------------------------------------------------- unfused L5 kernels
template <class R>
__global__ void k_node_backup(Params P, Nodes<R> Nd) {  // backup_current_velocity
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.nnodes) return;
    if (Nd.c[EXG_N_MASS][n] > R(0)) {
        Nd.c[EXG_N_MASS_OLD][n] = Nd.c[EXG_N_MASS][n];
        for (int d = 0; d < 3; ++d) Nd.c[EXG_N_DVEL + d][n] = Nd.c[EXG_N_VEL + d][n];
    }
}
template <class R>
__global__ void k_node_time_update(Params P, Nodes<R> Nd, double dt) {  // Nodal_Time_Update_Momentum
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.nnodes) return;
    double m = (double)Nd.c[EXG_N_MASS][n];
    for (int d = 0; d < 3; ++d) {
        if (m >= P.mass_tol)
            Nd.c[EXG_N_VEL + d][n] = (R)((double)Nd.c[EXG_N_VEL + d][n] + (double)Nd.c[EXG_N_FRC + d][n] / m * dt);
        else
            Nd.c[EXG_N_VEL + d][n] = R(0);
    }
}
template <class R>
__global__ void k_node_bcs(Params P, Nodes<R> Nd, NodeBCArgs bc, Ctl *ctl) {  // Apply_Nodal_BCs
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.nnodes) return;
    int i = (int)(n % P.nn[0]), j = (int)((n / P.nn[0]) % P.nn[1]), k = (int)(n / ((long long)P.nn[0] * P.nn[1]));
    if ((P.periodic[0] && i == P.nc[0]) || (P.periodic[1] && j == P.nc[1]) || (P.periodic[2] && k == P.nc[2])) return;
    unsigned status = 0;
    double m = (double)Nd.c[EXG_N_MASS][n];
    double v[3] = {(double)Nd.c[EXG_N_VEL][n], (double)Nd.c[EXG_N_VEL + 1][n], (double)Nd.c[EXG_N_VEL + 2][n]};
    node_bcs(P, bc, i, j, k, m, v, status);
    for (int d = 0; d < 3; ++d) {
        Nd.c[EXG_N_VEL + d][n] = (R)v[d];
        if (m > 0.0) Nd.c[EXG_N_DVEL + d][n] = (R)(v[d] - (double)Nd.c[EXG_N_DVEL + d][n]);
    }
    if (status) atomicOr(&ctl->status, status);
}

template <class R, int ORD>
__global__ void __launch_bounds__(kThreads) k_g2p_simple(Params P, Parts<R> A, Nodes<R> Nd, long long np, int upd_vel,
                                                         int upd_sr, double dt) {
    __shared__ SplineTables tab;
    load_tables(&tab);
    __syncthreads();
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= np || A.phase[p] != 0) return;
    GlobalNodes<R> na;
    for (int d = 0; d < 3; ++d) {
        na.v[d] = Nd.c[EXG_N_VEL + d];
        na.dv[d] = Nd.c[EXG_N_DVEL + d];
    }
    na.P = P;
    double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
    int iv[3];
    cell_of(P, x, iv);
    R v[3], vp[3], E[9], sr[6];
    for (int d = 0; d < 3; ++d) {
        v[d] = A.v[d][p];
        vp[d] = A.vp[d][p];
    }
    for (int q = 0; q < 9; ++q) E[q] = A.E[q][p];
    for (int c = 0; c < 6; ++c) sr[c] = A.sr[c][p];
    double jf = 1.0;
    g2p_particle<R, ORD>(tab, P, na, x, iv, upd_vel != 0, upd_sr != 0, v, vp, E, sr, dt, jf);
    if (sizeof(R) == 4 && upd_sr) A.J[p] *= jf;  // FP32 state: J kept in FP64 alongside F
    if (upd_vel)
        for (int d = 0; d < 3; ++d) {
            A.v[d][p] = v[d];
            A.vp[d][p] = vp[d];
        }
    if (upd_sr) {
        for (int q = 0; q < 9; ++q) A.E[q][p] = E[q];
        for (int c = 0; c < 6; ++c) A.sr[c][p] = sr[c];
    }
}

template <class R>
__global__ void k_move(Params P, Parts<R> A, NodeBCArgs bc, long long np, double dt, Ctl *ctl) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= np) return;
    unsigned status = 0;
    double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
    R v[3], vp[3];
    for (int d = 0; d < 3; ++d) {
        v[d] = A.v[d][p];
        vp[d] = A.vp[d][p];
    }
    move_particle<R>(P, bc, A.phase[p], x, v, vp, dt, status);
    for (int d = 0; d < 3; ++d) {
        A.x[d][p] = x[d];
        A.v[d][p] = v[d];
    }
    if (status) atomicOr(&ctl->status, status);
}

template <class R>
__global__ void k_vol_stress(Params P, Parts<R> A, const Material *mats, long long np, double dt, double asr,
                             int do_volume, int do_stress) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= np || A.phase[p] != 0) return;
    R E[9], sr[6], eps[6], sig[6];
    for (int q = 0; q < 9; ++q) E[q] = A.E[q][p];
    for (int c = 0; c < 6; ++c) {
        sr[c] = A.sr[c][p];
        eps[c] = A.eps[c][p];
        sig[c] = A.sig[c][p];
    }
    R vol = A.vol[p], rho = A.rho[p], pres = A.pres[p];
    double J = A.J[p];
    const Material mt = mats[A.mat[p]];
    if (do_stress && (mt.model < 0 || mt.model > 2)) return;
    volume_stress<R>(P, mt, E, A.vol0[p], A.mass[p], sr, eps, sig, vol, rho, J, pres, dt, asr, do_volume != 0,
                     do_stress != 0);
    if (do_volume) {
        A.vol[p] = vol;
        A.rho[p] = rho;
        A.J[p] = J;
    }
    if (do_stress) {
        for (int c = 0; c < 6; ++c) {
            A.eps[c][p] = eps[c];
            A.sig[c][p] = sig[c];
        }
        A.pres[p] = pres;
    }
}

// ---------------------------------------------------------------- thermal
// backup_current_temperature (nodal_data_ops.cpp:95-114),
// Nodal_Time_Update_Temperature (:500-527), store_delta_temperature
// (:409-430): one pass over the dense node arrays.
template <class R>
__global__ void k_temp_node_op(Params P, Nodes<R> Nd, int op, double dt) {
    long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.nnodes) return;
    const double mc = (double)Nd.c[EXG_N_MASS_SPHEAT][n];
    if (op == TN_BACKUP) {
        if (mc > 0.0) Nd.c[EXG_N_DELTA_TEMPERATURE][n] = Nd.c[EXG_N_TEMPERATURE][n];
    } else if (op == TN_TIME_UPDATE) {
        if (mc >= P.mass_tol)
            Nd.c[EXG_N_TEMPERATURE][n] =
                (R)((double)Nd.c[EXG_N_TEMPERATURE][n] + (double)Nd.c[EXG_N_SOURCE_TEMP][n] / mc * dt);
        else
            Nd.c[EXG_N_TEMPERATURE][n] = (R)(-P.Tref);
    } else {
        if (mc > 0.0)
            Nd.c[EXG_N_DELTA_TEMPERATURE][n] =
                (R)((double)Nd.c[EXG_N_TEMPERATURE][n] - (double)Nd.c[EXG_N_DELTA_TEMPERATURE][n]);
    }
}

// Domain-wall thermal BCs, nodal_bcs_temperature (nodal_data_ops.cpp:786-910)
// then apply_udf_nodal_bcs_temperature (:1296-1446).  Both are in-place
// sweeps in node order (x fastest): a node on a high face reads its inward
// neighbour after that neighbour's own update in the same sweep, a node on a
// low face reads it before.  Only the last direction that writes a node
// decides its value, so the sweep result of a node is a chain of at most
// three links (one per high face), each a function of the next node's
// value; every thread evaluates its node's chain from the values stored
// before the pass, which gives the sweep result without ordering.
struct TLink {
    signed char dir, side, kind;
    double a, b;  // wall constants of the link (value, second value)
};

template <class R>
struct TempView {
    const R *T, *mc, *mk, *m;
    bool mask;  // fused step: nodes below the mass tolerance hold 0 K before the pass
    double mass_tol, Tref;
    __device__ __forceinline__ double pre(long long n) const {
        if (mask && !((double)mc[n] >= mass_tol)) return -Tref;
        return (double)T[n];
    }
    // specific conductance k = (m k) / m, 1 on massless nodes
    __device__ __forceinline__ double kn(long long n) const {
        const double mm = (double)m[n];
        return (mm > 0.0) ? (double)mk[n] / mm : 1.0;
    }
};

__device__ __forceinline__ bool temp_wall_link(const Params &P, const int id[3], TLink &L) {
    bool applied = false, any = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const bool lo = id[d] == 0;
        const bool hi = !lo && id[d] == P.nc[d];
        if (!lo && !hi) continue;
        const int bc = lo ? P.bclo_temp[d] : P.bchi_temp[d];
        const bool writes = bc == EXG_BCT_ISOTHERMAL || bc == EXG_BCT_USERFLUX || bc == EXG_BCT_CONVECTION ||
                            (bc == EXG_BCT_ADIABATIC && !applied);
        if (bc == EXG_BCT_PERIODIC || writes) applied = true;
        if (!writes) continue;
        any = true;
        L.dir = (signed char)d;
        L.side = hi ? 1 : 0;
        L.kind = (signed char)bc;
        L.a = L.b = 0.0;
        if (bc == EXG_BCT_ISOTHERMAL) {
            L.a = (lo ? P.Twall_lo[d] : P.Twall_hi[d]) - P.Tref;
        } else if (bc == EXG_BCT_USERFLUX) {
            L.a = lo ? P.qflux_lo[d] : P.qflux_hi[d];
        } else if (bc == EXG_BCT_CONVECTION) {
            L.a = lo ? P.hc_lo[d] : P.hc_hi[d];
            L.b = (lo ? P.Tinf_lo[d] : P.Tinf_hi[d]) - P.Tref;
        }
    }
    return any;
}

__device__ __forceinline__ bool temp_udf_link(const Params &P, const NodeBCArgs &bc, const int id[3], TLink &L) {
    bool any = false;
#pragma unroll
    for (int dir = 0; dir < 3; ++dir) {
        const double *tab = nullptr;
        int code = -1, side = 0;
        if (id[dir] == 0 && bc.udfT[0][dir]) {
            tab = bc.udfT[0][dir];
            code = P.bclo_temp[dir];
        } else if (id[dir] == P.nc[dir] && bc.udfT[1][dir]) {
            tab = bc.udfT[1][dir];
            code = P.bchi_temp[dir];
            side = 1;
        }
        if (!tab) continue;
        if (code != EXG_BCT_ISOTHERMAL && code != EXG_BCT_USERFLUX && code != EXG_BCT_CONVECTION) continue;
        const int p0 = (dir == 0) ? 1 : 0, p1 = (dir == 2) ? 1 : 2;
        const long long f = ((long long)id[p0] * (P.nc[p1] + 1) + id[p1]) * 2;
        any = true;
        L.dir = (signed char)dir;
        L.side = (signed char)side;
        L.kind = (signed char)code;
        // temperatures (isothermal value, convective T_inf) relative to Tref
        L.a = tab[f] - (code == EXG_BCT_ISOTHERMAL ? P.Tref : 0.0);
        L.b = tab[f + 1] - (code == EXG_BCT_CONVECTION ? P.Tref : 0.0);
    }
    return any;
}

// Value written by one link given its neighbour's value.
__device__ __forceinline__ double temp_link_apply(const Params &P, const TLink &L, double Tnb, double kn) {
    const double h = P.dx[L.dir];
    if (L.kind == EXG_BCT_ISOTHERMAL) return L.a;
    if (L.kind == EXG_BCT_ADIABATIC) return Tnb;
    if (L.kind == EXG_BCT_USERFLUX) return Tnb + L.a * h / kn;
    const double Bi = L.a * h / kn;
    return (Tnb + Bi * L.b) / (1.0 + Bi);
}

__device__ __forceinline__ long long node_lin(const Params &P, const int id[3]) {
    return ((long long)id[2] * P.nn[1] + id[1]) * P.nn[0] + id[0];
}

// Result of the wall sweep at node id.
template <class R>
__device__ double temp_wall_value(const Params &P, const TempView<R> &tv, const int id0[3], unsigned &status) {
    TLink L[3];
    long long ln[3];
    int nl = 0;
    int id[3] = {id0[0], id0[1], id0[2]};
    double val = 0.0;
    for (int it = 0;; ++it) {
        TLink l;
        const long long n = node_lin(P, id);
        if (!temp_wall_link(P, id, l)) {
            val = tv.pre(n);
            break;
        }
        if (l.kind == EXG_BCT_ISOTHERMAL) {
            val = l.a;
            break;
        }
        int nb[3] = {id[0], id[1], id[2]};
        nb[l.dir] += l.side ? -1 : 1;
        if (!l.side) {  // low face: the neighbour is swept later
            val = temp_link_apply(P, l, tv.pre(node_lin(P, nb)), tv.kn(n));
            break;
        }
        if (nl == 3) {  // at most three high faces: unreachable
            status |= ST_BC;
            break;
        }
        L[nl] = l;
        ln[nl++] = n;
        id[0] = nb[0];
        id[1] = nb[1];
        id[2] = nb[2];
    }
    for (int k = nl - 1; k >= 0; --k) val = temp_link_apply(P, L[k], val, tv.kn(ln[k]));
    return val;
}

// Result of the wall sweep followed by the UDF sweep at node id.
template <class R>
__device__ double temp_face_value(const Params &P, const NodeBCArgs &bc, const TempView<R> &tv, const int id0[3],
                                  bool walls, bool udf, unsigned &status) {
    TLink L[3];
    long long ln[3];
    int nl = 0;
    int id[3] = {id0[0], id0[1], id0[2]};
    double val = 0.0;
    for (int it = 0;; ++it) {
        TLink l;
        const long long n = node_lin(P, id);
        if (!udf || !temp_udf_link(P, bc, id, l)) {
            val = walls ? temp_wall_value<R>(P, tv, id, status) : tv.pre(n);
            break;
        }
        if (l.kind == EXG_BCT_ISOTHERMAL) {
            val = l.a;
            break;
        }
        int nb[3] = {id[0], id[1], id[2]};
        nb[l.dir] += l.side ? -1 : 1;
        if (!l.side) {
            const double before = walls ? temp_wall_value<R>(P, tv, nb, status) : tv.pre(node_lin(P, nb));
            val = temp_link_apply(P, l, before, tv.kn(n));
            break;
        }
        if (nl == 3) {
            status |= ST_BC;
            break;
        }
        L[nl] = l;
        ln[nl++] = n;
        id[0] = nb[0];
        id[1] = nb[1];
        id[2] = nb[2];
    }
    for (int k = nl - 1; k >= 0; --k) val = temp_link_apply(P, L[k], val, tv.kn(ln[k]));
    return val;
}

// Face-node entries: for each non-periodic axis d and side, the owned nodes
// of that face; a node on an edge or corner appears once per face and every
// entry computes the same value.
__device__ __forceinline__ bool face_entry(const Params &P, long long e, int id[3]) {
    for (int d = 0; d < 3; ++d) {
        if (P.periodic[d]) continue;
        const int p0 = (d == 0) ? 1 : 0, p1 = (d == 2) ? 1 : 2;
        const long long n0 = P.periodic[p0] ? P.nc[p0] : P.nc[p0] + 1;
        const long long n1 = P.periodic[p1] ? P.nc[p1] : P.nc[p1] + 1;
        const long long per = n0 * n1;
        if (e < 2 * per) {
            const int side = (int)(e / per);
            const long long r = e % per;
            id[d] = side ? P.nc[d] : 0;
            id[p0] = (int)(r % n0);
            id[p1] = (int)(r / n0);
            return true;
        }
        e -= 2 * per;
    }
    return false;
}

template <class R>
__global__ void k_temp_faces(Params P, Nodes<R> Nd, NodeBCArgs bc, double *out, long long nface, int walls, int mask,
                             int udf, Ctl *ctl) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nface) return;
    int id[3];
    if (!face_entry(P, e, id)) return;
    TempView<R> tv{Nd.c[EXG_N_TEMPERATURE], Nd.c[EXG_N_MASS_SPHEAT], Nd.c[EXG_N_MASS_COND], Nd.c[EXG_N_MASS],
                   mask != 0, P.mass_tol, P.Tref};
    unsigned status = 0;
    out[e] = temp_face_value<R>(P, bc, tv, id, walls != 0, udf != 0, status);
    if (status) atomicOr(&ctl->status, status);
}

template <class R>
__global__ void k_temp_faces_store(Params P, Nodes<R> Nd, const double *in, long long nface) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= nface) return;
    int id[3];
    if (!face_entry(P, e, id)) return;
    Nd.c[EXG_N_TEMPERATURE][node_lin(P, id)] = (R)in[e];
}

// nodal_levelset_bcs_temperature (nodal_data_ops.cpp:235-349) for one body:
// nodes inside the body (phi < 0) that carry heat capacity take the wall
// temperature, or the flux / convective value from the neighbour one step
// along the dominant axis of the outward normal, read as it was before the
// body's pass.  Writes every node of dst.
template <class R>
__global__ void k_temp_levelset(Params P, Nodes<R> Nd, const double *phi, int b, const R *src, R *dst) {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.nnodes) return;
    const int id[3] = {(int)(n % P.nn[0]), (int)((n / P.nn[0]) % P.nn[1]), (int)(n / ((long long)P.nn[0] * P.nn[1]))};
    R out = src[n];
    bool owned = true;
    for (int d = 0; d < 3; ++d) owned = owned && !(P.periodic[d] && id[d] == P.nc[d]);
    if (owned && (double)Nd.c[EXG_N_MASS_SPHEAT][n] > 0.0) {
        const double xn[3] = {P.plo[0] + id[0] * P.dx[0], P.plo[1] + id[1] * P.dx[1], P.plo[2] + id[2] * P.dx[2]};
        double lv, nd[3];
        ls_sample(P, phi, xn, lv, nd);
        const double gm = sqrt(nd[0] * nd[0] + nd[1] * nd[1] + nd[2] * nd[2]);
        if (lv < 0.0 && !(gm < 1.0e-10)) {
            for (int d = 0; d < 3; ++d) nd[d] /= gm;
            const Body &bd = P.body[b];
            if (bd.temp_bc == 1) {
                out = (R)(bd.T_wall - P.Tref);
            } else if (bd.temp_bc == 3 || bd.temp_bc == 4) {
                int dd = 0;
                for (int d = 1; d < 3; ++d)
                    if (fabs(nd[d]) > fabs(nd[dd])) dd = d;
                int nb[3] = {id[0], id[1], id[2]};
                nb[dd] += (nd[dd] > 0.0) ? 1 : -1;
                const double mm = (double)Nd.c[EXG_N_MASS][n];
                const double kn = (mm > 0.0) ? (double)Nd.c[EXG_N_MASS_COND][n] / mm : 1.0;
                const long long q = node_index(P, nb[0], nb[1], nb[2]);
                const double Tnb = q < 0 ? -P.Tref : (double)src[q];  // ghost nodes hold 0 K
                if (bd.temp_bc == 3) {
                    out = (R)(Tnb + bd.heat_flux * P.dx[dd] / kn);
                } else {
                    const double Bi = bd.h_conv * P.dx[dd] / kn;
                    out = (R)((Tnb + Bi * (bd.T_inf - P.Tref)) / (1.0 + Bi));
                }
            }
        }
    }
    dst[n] = out;
}

// interpolate_from_grid_temperature (mpm_particle_grid_ops.cpp:1129-1270):
// T += interpolated nodal temperature increment (scheme of the x order, as
// the reference selects it) and q = -k grad T from the nodal temperatures.
template <class R, int ORD>
__global__ void __launch_bounds__(kThreads) k_g2p_temp(Params P, Parts<R> A, Nodes<R> Nd, long long np, int upd_T,
                                                       int upd_q) {
    __shared__ SplineTables tab;
    load_tables(&tab);
    __syncthreads();
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= np || A.phase[p] != 0) return;
    const double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
    int iv[3];
    cell_of(P, x, iv);
    if (upd_T) {
        const R *dT = Nd.c[EXG_N_DELTA_TEMPERATURE];
        R wx[4], wy[4], wz[4];
        interp_axis<R>(tab, P, P.order[0], 0, x[0], iv[0], wx);
        interp_axis<R>(tab, P, P.order[0], 1, x[1], iv[1], wy);
        interp_axis<R>(tab, P, P.order[0], 2, x[2], iv[2], wz);
        R acc = R(0);
        for (int sz = 0; sz < 4; ++sz)
            for (int sy = 0; sy < 4; ++sy)
                for (int sx = 0; sx < 4; ++sx) {
                    const R N = wx[sx] * wy[sy] * wz[sz];
                    if (N == R(0)) continue;
                    const long long q = node_index(P, iv[0] - 1 + sx, iv[1] - 1 + sy, iv[2] - 1 + sz);
                    if (q >= 0) acc += N * dT[q];
                }
        A.T[p] = A.T[p] + (double)acc;
    }
    if (upd_q) {
        constexpr int W = Stc<ORD>::W, LO = Stc<ORD>::LO;
        const R *Tn = Nd.c[EXG_N_TEMPERATURE];
        AxisW<R, W> ax, ay, az;
        axis_weights<R, W, LO>(tab, P, 0, x[0], iv[0], ax);
        axis_weights<R, W, LO>(tab, P, 1, x[1], iv[1], ay);
        axis_weights<R, W, LO>(tab, P, 2, x[2], iv[2], az);
        R g[3] = {R(0), R(0), R(0)};
        for (int sz = 0; sz < W; ++sz)
            for (int sy = 0; sy < W; ++sy)
                for (int sx = 0; sx < W; ++sx) {
                    const R gx = ax.dw[sx] * ay.w[sy] * az.w[sz], gy = ax.w[sx] * ay.dw[sy] * az.w[sz],
                            gz = ax.w[sx] * ay.w[sy] * az.dw[sz];
                    if (gx == R(0) && gy == R(0) && gz == R(0)) continue;
                    const long long q = node_index(P, iv[0] + LO + sx, iv[1] + LO + sy, iv[2] + LO + sz);
                    const R t = q >= 0 ? Tn[q] : R(0);
                    g[0] += t * gx;
                    g[1] += t * gy;
                    g[2] += t * gz;
                }
        const R k = A.kc[p];
        for (int d = 0; d < 3; ++d) A.q[d][p] = -k * g[d];
    }
}

// Do_All_Diagnostics reductions (mpm_diagnostics.cpp:23-216) as one pass with
// a fixed-shape tree: per-block partials in FP64, summed in block order by a
// second single-block pass, so the result is deterministic.
constexpr int kDiagN = 16;  // tke tse mass mom3 mvm min3 max3 np
template <class R>
__global__ void __launch_bounds__(kThreads) k_diag_partial(Params P, Parts<R> A, long long np, double *part) {
    __shared__ double sh[kDiagN][kThreads];
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double a[kDiagN];
    for (int c = 0; c < kDiagN; ++c) a[c] = 0.0;
    a[9] = a[10] = a[11] = 1.7976931348623157e308;
    a[12] = a[13] = a[14] = -1.7976931348623157e308;
    if (p < np) {
        double x[3] = {A.x[0][p], A.x[1][p], A.x[2][p]};
        int iv[3];
        cell_of(P, x, iv);
        bool in = true;
        for (int d = 0; d < 3; ++d) in = in && iv[d] >= 0 && iv[d] < P.nc[d];
        if (in) {
            double m = A.mass[p];
            double v[3] = {(double)A.v[0][p], (double)A.v[1][p], (double)A.v[2][p]};
            double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            a[0] = 0.5 * m * v2;
            double s[6], e[6];
            for (int c = 0; c < 6; ++c) {
                s[c] = A.sig[c][p];
                e[c] = A.eps[c][p];
            }
            double se = s[0] * e[0] + s[3] * e[3] + s[5] * e[5] + 2.0 * (s[1] * e[1] + s[4] * e[4] + s[2] * e[2]);
            a[1] = 0.5 * (double)A.vol[p] * se;
            a[2] = m;
            for (int d = 0; d < 3; ++d) a[3 + d] = m * v[d];
            a[6] = m * sqrt(v2);
            for (int d = 0; d < 3; ++d) {
                a[9 + d] = x[d];
                a[12 + d] = x[d];
            }
            a[15] = 1.0;
        }
    }
    for (int c = 0; c < kDiagN; ++c) sh[c][threadIdx.x] = a[c];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int c = 0; c < kDiagN; ++c) {
                double o = sh[c][threadIdx.x + s];
                if (c >= 9 && c < 12)
                    sh[c][threadIdx.x] = fmin(sh[c][threadIdx.x], o);
                else if (c >= 12 && c < 15)
                    sh[c][threadIdx.x] = fmax(sh[c][threadIdx.x], o);
                else
                    sh[c][threadIdx.x] += o;
            }
        __syncthreads();
    }
    if (threadIdx.x < kDiagN) part[(long long)blockIdx.x * kDiagN + threadIdx.x] = sh[threadIdx.x][0];
}
__global__ void k_diag_final(const double *part, int nblk, double *out) {
    int c = threadIdx.x;
    if (c >= kDiagN) return;
    double acc = (c >= 9 && c < 12) ? 1.7976931348623157e308 : ((c >= 12 && c < 15) ? -1.7976931348623157e308 : 0.0);
    for (int b = 0; b < nblk; ++b) {
        double v = part[(long long)b * kDiagN + c];
        if (c >= 9 && c < 12)
            acc = fmin(acc, v);
        else if (c >= 12 && c < 15)
            acc = fmax(acc, v);
        else
            acc += v;
    }
    out[c] = acc;
}

// ---------------------------------------------------------------- batched scenes
// Many independent scenes (each a context with its own grid, particles,
// control block and buffers) advance with ONE launch of each hot kernel: the
// items are the concatenation of every scene's tile list, taken dynamically;
// a block reads the item's scene descriptor in place (read-only global
// memory, so its fields stay in registers and the L1 across the tile) and
// runs the same tile code as the single-scene kernels.
template <class R>
struct SceneDesc {
    Params P;
    Parts<R> A, Bo;
    Nodes<R> N;
    NodeBCArgs bc;
    const Material *mats;
    const int *active, *start, *count, *cell_start, *touched, *slot;
    const int32_t *perm;
    long long *staging;
    Ctl *ctl;
};

// Largest s with pre[s] <= i (pre[0] = 0, pre ascending).
__device__ __forceinline__ int scene_of(const int *pre, int ns, int i) {
    int lo = 0, hi = ns;  // invariant: pre[lo] <= i < pre[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= i)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Prefix sums of the scenes' active and touched tile counts; resets the
// batch's tile counters.  One block.
__global__ void k_batch_plan(BatchCtl *b, Ctl *const *ctls) {
    __shared__ int sh[34];
    __shared__ int ca, ct;
    const int ns = b->nscenes;
    if (threadIdx.x == 0) {
        ca = ct = 0;
        b->next_p2g = b->next_nodes = b->next_g2p = b->next_sort = 0;
    }
    __syncthreads();
    for (int base = 0; base < ns; base += blockDim.x) {
        const int s = base + threadIdx.x;
        const int na = s < ns ? ctls[s]->n_active_tiles : 0;
        const int nt = s < ns ? ctls[s]->n_touched_tiles : 0;
        int ta, tt;
        const int ea = block_exclusive_scan(na, &ta, sh);
        const int et = block_exclusive_scan(nt, &tt, sh);
        if (s < ns) {
            b->pre_active[s] = ca + ea;
            b->pre_touched[s] = ct + et;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            ca += ta;
            ct += tt;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        b->pre_active[ns] = ca;
        b->pre_touched[ns] = ct;
    }
}

#if defined(EXG_R_FP64)
// ---- batched sort and bookkeeping: one launch of each kernel for all
// scenes, running the single-scene bodies, so a batched scene is sorted
// exactly as when stepped alone.  Per-particle kernels map each block to one
// scene (BatchCtl::pre_blocks), so no warp mixes scenes; per-tile kernels map
// threads through BatchCtl::pre_tiles.

// Step start: the step's P2G bounds (those of the last G2P), dt and the
// accumulator reset (k_dt_finalize) of scene i < nscenes by thread i; zeroed
// tile counts of every scene.
__global__ void k_bb_start(const SortDesc *__restrict__ d, const BatchCtl *__restrict__ b) {
    const int ns = b->nscenes, tot = b->pre_tiles[ns];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ns) {
        const SortDesc &x = d[i];
        for (int c = 0; c < CH_ALL; ++c) x.bounds_cur[c] = x.ctl->bound_bits[c];
        dt_finalize_body(x.P, x.ctl, 1);
    }
    if (i < tot) {
        const int s = scene_of(b->pre_tiles, ns, i);
        const int t = i - b->pre_tiles[s];
        d[s].tile_count[t] = 0;
        d[s].tile_fill[t] = 0;
    }
}

__global__ void __launch_bounds__(kBatchThreads) k_bb_keys(const SortDesc *__restrict__ d,
                                                            const BatchCtl *__restrict__ b) {
    const int s = scene_of(b->pre_blocks, b->nscenes, blockIdx.x);
    const SortDesc &x = d[s];
    const long long i = (long long)(blockIdx.x - b->pre_blocks[s]) * blockDim.x + threadIdx.x;
    keys_body(x.P, x.x[0], x.x[1], x.x[2], x.np, x.key, x.tile_count, x.ctl, 1, i);
}

__global__ void k_bb_tile_scan(const SortDesc *__restrict__ d) {
    const SortDesc &x = d[blockIdx.x];
    tile_scan_block((int)x.P.ntiles, x.tile_count, x.tile_start, x.active, x.slot, x.item_start, x.ctl);
}

__global__ void __launch_bounds__(kBatchThreads) k_bb_scatter(const SortDesc *__restrict__ d,
                                                               const BatchCtl *__restrict__ b) {
    const int s = scene_of(b->pre_blocks, b->nscenes, blockIdx.x);
    const SortDesc &x = d[s];
    const long long i = (long long)(blockIdx.x - b->pre_blocks[s]) * blockDim.x + threadIdx.x;
    scatter_body(x.np, x.key, 3 * x.P.tshift, x.tile_start, x.tile_fill, x.bucket, i);
}

// Persistent blocks over the concatenated active-tile lists (the tile order
// of k_batch_plan's prefix sums), taken from a device counter.
__global__ void __launch_bounds__(kThreads) k_bb_tile_sort(const SortDesc *__restrict__ d, BatchCtl *b, int ncell) {
    extern __shared__ int sm[];
    __shared__ int s_item, s_scene;
    const int ns = b->nscenes, total = b->pre_active[ns];
    for (;;) {
        if (threadIdx.x == 0) {
            const int i = atomicAdd(&b->next_sort, 1);
            s_item = i;
            s_scene = i < total ? scene_of(b->pre_active, ns, i) : -1;
        }
        __syncthreads();
        const int i = s_item, s = s_scene;
        if (i >= total) break;
        const SortDesc &x = d[s];
        tile_sort_item(sm, x.active, x.tile_start, x.tile_count, x.key, x.bucket, x.bucket + x.cap, x.perm,
                       x.cell_start, ncell, x.ctl, i - b->pre_active[s]);
    }
}

__global__ void k_bb_touched(const SortDesc *__restrict__ d, const BatchCtl *__restrict__ b) {
    const int ns = b->nscenes, i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b->pre_tiles[ns]) return;
    const int s = scene_of(b->pre_tiles, ns, i);
    const SortDesc &x = d[s];
    touched_body(x.P, x.tile_count, x.touched, x.touched_step, x.ctl, i - b->pre_tiles[s]);
}

// One block per scene, one thread per fixed-point channel.
__global__ void k_bb_scales(const SortDesc *__restrict__ d, int stencil_cells, int bits) {
    const SortDesc &x = d[blockIdx.x];
    scales_body(x.ctl, stencil_cells, bits, x.bounds_cur, threadIdx.x);
}

#endif  // EXG_R_FP64

__global__ void k_bb_time_advance(const SortDesc *__restrict__ d, int ns) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ns) return;
    Ctl *ctl = d[s].ctl;
    ctl->time += ctl->dt;
    ctl->steps += 1;
}

// Particles outside the domain of every scene after the batched G2P (see
// k_copy_lost).
template <class R>
__global__ void __launch_bounds__(kBatchThreads) k_bb_copy_lost(const SceneDesc<R> *__restrict__ dr,
                                                                 const SortDesc *__restrict__ d,
                                                                 const BatchCtl *__restrict__ b, int temp) {
    const int s = scene_of(b->pre_blocks, b->nscenes, blockIdx.x);
    const SortDesc &x = d[s];
    Ctl *ctl = x.ctl;
    if (ctl->lost == 0) return;
    const long long i = (long long)(blockIdx.x - b->pre_blocks[s]) * blockDim.x + threadIdx.x;
    if (i >= x.np || x.key[i] != 0xFFFFFFFFu) return;
    const long long j = ctl->n_sorted + (long long)atomicAdd(&ctl->lost_fill, 1ull);
    Parts<R> Bo = dr[s].Bo;
    copy_particle<R>(dr[s].A, i, Bo, j, temp != 0);
}

template <class R, int ORD, bool THERM>
__global__ void __launch_bounds__(P2GCfg<R, ORD, THERM>::THREADS, P2GCfg<R, ORD, THERM>::MINB)
    k_p2g_batch(const SceneDesc<R> *__restrict__ descs, BatchCtl *b, int B3) {
    constexpr int NCH = THERM ? CH_ALL : CH_MOM_END;
    __shared__ int s_item, s_scene;
    extern __shared__ __align__(16) unsigned char smraw[];
    SplineTables *tab = reinterpret_cast<SplineTables *>(smraw);
    unsigned *acc_lo = reinterpret_cast<unsigned *>(smraw + ((sizeof(SplineTables) + 15) & ~15));
    int *acc_hi = reinterpret_cast<int *>(acc_lo + NCH * B3 * fx_lo_words<R>());
    load_tables(tab);
    const int ns = b->nscenes, total = b->pre_active[ns];
    int cur = -1;
    R sc[NCH], grav[3];
    for (;;) {
        if (threadIdx.x == 0) {
            const int i = atomicAdd(&b->next_p2g, 1);
            s_item = i;
            s_scene = i < total ? scene_of(b->pre_active, ns, i) : -1;
        }
        fx_zero<R>(acc_lo, acc_hi, NCH * B3);
        __syncthreads();
        const int i = s_item, s = s_scene;
        if (i >= total) break;
        const SceneDesc<R> &sd = descs[s];
        if (s != cur) {
            cur = s;
#pragma unroll
            for (int c = 0; c < NCH; ++c) sc[c] = (R)sd.ctl->scale[c];
#pragma unroll
            for (int d = 0; d < 3; ++d) grav[d] = (R)sd.P.gravity[d];
        }
        if constexpr (P2GCfg<R, ORD, THERM>::FACT)
            p2g_tile_factorized<R, ORD, P2GCfg<R, ORD, THERM>::ROWS, P2GCfg<R, ORD, THERM>::MAP>(
                tab, acc_lo, acc_hi, sd.P, sd.A, sd.active, sd.start, sd.cell_start, sd.perm, sd.staging, sc, grav,
                i - b->pre_active[s]);
        else
            p2g_tile<R, ORD, THERM>(tab, acc_lo, acc_hi, sd.P, sd.A, sd.active, sd.start, sd.cell_start, sd.perm,
                                    sd.staging, sc, grav, i - b->pre_active[s]);
    }
}

template <class R, bool THERM>
__global__ void __launch_bounds__(kThreads, EXG_NODES_MINB) k_nodes_batch(const SceneDesc<R> *__restrict__ descs, BatchCtl *b, int mode,
                                                          int flags) {
    constexpr int NCH = THERM ? CH_ALL : CH_MOM_END;
    __shared__ int s_item, s_scene;
    const int ns = b->nscenes, total = b->pre_touched[ns];
    int cur = -1;
    unsigned status = 0;
    double isc[NCH], dt = 0.0;
    for (;;) {
        if (threadIdx.x == 0) {
            const int i = atomicAdd(&b->next_nodes, 1);
            s_item = i;
            s_scene = i < total ? scene_of(b->pre_touched, ns, i) : -1;
        }
        __syncthreads();
        const int i = s_item, s = s_scene;
        if (i >= total) break;
        const SceneDesc<R> &sd = descs[s];
        if (s != cur) {
            if (cur >= 0 && status) atomicOr(&descs[cur].ctl->status, status);
            status = 0;
            cur = s;
#pragma unroll
            for (int c = 0; c < NCH; ++c) isc[c] = sd.ctl->inv_scale[c];
            dt = sd.ctl->dt;
        }
        nodes_tile<R, THERM>(sd.P, sd.N, sd.bc, sd.touched, sd.slot, sd.staging, isc, dt, mode, flags,
                             i - b->pre_touched[s], status);
        __syncthreads();
    }
    if (cur >= 0 && status) atomicOr(&descs[cur].ctl->status, status);
}

template <class R, int ORD, bool LEAN>
__global__ void __launch_bounds__(EXG_G2P_THREADS, EXG_G2P_MINB)
    k_g2p_batch(const SceneDesc<R> *__restrict__ descs, BatchCtl *b, int mode) {
    __shared__ int s_item, s_scene;
    extern __shared__ __align__(16) unsigned char smraw[];
    SplineTables *tab = reinterpret_cast<SplineTables *>(smraw);
    R *nb = reinterpret_cast<R *>(smraw + ((sizeof(SplineTables) + 15) & ~15));
    load_tables(tab);
    const int ns = b->nscenes, total = b->pre_active[ns];
    const bool upd_vel = (mode != GM_STRAIN);
    int cur = -1;
    unsigned status = 0;
    double dt = 0.0, asr = 0.0;
    float run_b[CH_ALL];
    double run_speed = 0.0;
    bool red = false;
    // the reductions of a scene go to its control block when the block moves
    // on to another scene, and at the end
    auto flush = [&](const SceneDesc<R> &sd) {
        Ctl *ctl = sd.ctl;
        if (mode != GM_VEL) {
            double rb[CH_ALL];
#pragma unroll
            for (int c = 0; c < CH_ALL; ++c) rb[c] = (double)run_b[c];
            block_reduce_push(&ctl->bound_bits[0], &ctl->dtmin_bits, rb, sd.P.dxmin / run_speed, red);
        }
        if (status) atomicOr(&ctl->status, status);
        __syncthreads();
    };
    for (;;) {
        if (threadIdx.x == 0) {
            const int i = atomicAdd(&b->next_g2p, 1);
            s_item = i;
            s_scene = i < total ? scene_of(b->pre_active, ns, i) : -1;
        }
        __syncthreads();
        const int i = s_item, s = s_scene;
        if (i >= total) break;
        const SceneDesc<R> &sd = descs[s];
        if (s != cur) {
            if (cur >= 0) flush(descs[cur]);
            cur = s;
            dt = sd.ctl->dt;
            const double time = sd.ctl->time;
            asr = (time < sd.P.applied_sr_time) ? sd.P.applied_sr : 0.0;
#pragma unroll
            for (int c = 0; c < CH_ALL; ++c) run_b[c] = 0.0f;
            run_speed = 0.0;
            red = false;
            status = 0;
        }
        g2p_tile<R, ORD, LEAN>(tab, nb, sd.P, sd.A, sd.Bo, sd.N, sd.bc, sd.mats, sd.active, sd.start, sd.count, sd.perm, mode,
                         i - b->pre_active[s], dt, asr, upd_vel, run_b, run_speed, red, status);
    }
    if (cur >= 0) flush(descs[cur]);
}

template <class R>
__global__ void k_fill(R *a, long long n, double value) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) a[i] = (R)value;
}

// ---------------------------------------------------------------- host transfers
// Particle fields cross PCIe as the caller's FP64 arrays; the precision
// conversion and the return to upload order run here.
template <class R>
__global__ void k_from_f64(const double *src, R *dst, long long n, double sub) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (R)(src[i] - sub);
}
// pid == nullptr: the field is stored in upload order already
template <class R>
__global__ void k_to_f64_unperm(const R *src, const int32_t *pid, double *dst, long long n, double add) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[pid ? pid[i] : i] = (double)src[i] + add;
}
template <class T>
__global__ void k_unperm_i32(const T *src, const int32_t *pid, int32_t *dst, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) dst[pid ? pid[i] : i] = (int32_t)src[i];
}

}  // namespace

// ====================================================================== launchers
static int nblocks(long long n, int t = kThreads) { return (int)((n + t - 1) / t); }

// Grid of a persistent kernel: every SM filled to its occupancy limit.
template <class K>
static int persistent_grid(K kern, size_t smem, int threads = kThreads) {
    int dev = 0, nsm = 0, per = 0;
    EXG_CUDA_OK(cudaGetDevice(&dev));
    EXG_CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    EXG_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem));
    if (per < 1) per = 1;
    return nsm * per;
}

static NodeBCArgs make_bc(Ctx &c) {
    NodeBCArgs bc;
    for (int s = 0; s < 2; ++s)
        for (int d = 0; d < 3; ++d) {
            bc.udf[s][d] = c.udf_tab[s][d];
            bc.udfT[s][d] = c.udfT_tab[s][d];
        }
    for (int b = 0; b < kMaxBodies; ++b) bc.ls[b] = c.ls[b];
    return bc;
}

#if defined(EXG_R_FP64)
void launch_keys(Ctx &c) {
    EXG_CUDA_OK(cudaMemsetAsync(c.sb.tile_count, 0, sizeof(int) * c.P.ntiles, c.stream));
    EXG_CUDA_OK(cudaMemsetAsync(c.sb.tile_fill, 0, sizeof(int) * c.P.ntiles, c.stream));
    double **x = c.precision == EXG_PREC_FP64 ? c.A<double>().x : c.A<float>().x;
    if (c.np > 0)
        k_keys<<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, x[0], x[1], x[2], c.np, c.sb.key, c.sb.tile_count, c.ctl,
                                                         1);
    EXG_CUDA_OK(cudaGetLastError());
}

void launch_sort_rest(Ctx &c, bool touched_list) {
    k_tile_scan<<<1, 1024, 0, c.stream>>>((int)c.P.ntiles, c.sb.tile_count, c.sb.tile_start, c.sb.active, c.sb.slot,
                                          c.sb.item_start, c.ctl);
    if (c.np > 0)
        k_scatter<<<nblocks(c.np), kThreads, 0, c.stream>>>(c.np, c.sb.key, 3 * c.P.tshift, c.sb.tile_start,
                                                            c.sb.tile_fill, c.sb.bucket);
    const int ncell = c.P.T * c.P.T * c.P.T;
    size_t sm = sizeof(int) * (3 * ncell + kSortCap);
    EXG_CUDA_OK(cudaFuncSetAttribute(k_tile_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    static int sgrid = 0;
    if (!sgrid) sgrid = persistent_grid(k_tile_sort, sm);
    // no more blocks than the scene has tiles (small scenes of a batch)
    const int tgrid = (int)std::min<long long>(sgrid, c.P.ntiles);
    k_tile_sort<<<tgrid, kThreads, sm, c.stream>>>(c.sb.active, c.sb.tile_start, c.sb.tile_count, c.sb.key,
                                                    c.sb.bucket, c.sb.bucket + c.cap, c.sb.perm, c.sb.cell_start, ncell,
                                                    c.ctl);
    if (touched_list)
        k_touched<<<nblocks(c.P.ntiles), kThreads, 0, c.stream>>>(c.P, c.sb.tile_count, c.sb.touched,
                                                                  c.sb.touched_step, c.ctl);
    EXG_CUDA_OK(cudaGetLastError());
}

void launch_dt_finalize(Ctx &c, bool reset) {
    k_dt_finalize<<<1, 1, 0, c.stream>>>(c.P, c.ctl, reset ? 1 : 0);
    EXG_CUDA_OK(cudaGetLastError());
}

void launch_scales_from(Ctx &c, const unsigned long long *bounds) {
    const int W = (c.P.uniform_order == 1) ? 2 : (c.P.dual ? 3 : 4);
    k_scales<<<1, 32, 0, c.stream>>>(c.ctl, W * W * W, c.precision == EXG_PREC_FP64 ? kFxBits64 : kFxBits32, bounds);
    EXG_CUDA_OK(cudaGetLastError());
}

void launch_reset_accum(Ctx &c, unsigned long long *bounds, unsigned long long *dtmin) {
    k_reset_accum<<<1, 32, 0, c.stream>>>(bounds, dtmin);
    EXG_CUDA_OK(cudaGetLastError());
}

void launch_time_advance(Ctx &c) {
    k_time_advance<<<1, 1, 0, c.stream>>>(c.ctl);
    EXG_CUDA_OK(cudaGetLastError());
}

void launch_node_reset(Ctx &c) {
    const size_t esz = c.precision == EXG_PREC_FP64 ? 8 : 4;
    for (void *p : c.node_allocs) EXG_CUDA_OK(cudaMemsetAsync(p, 0, esz * c.P.nnodes, c.stream));
}
#endif

// ---- precision-specific launchers
void EXG_SFX(launch_state_reduce)(Ctx &c, unsigned long long *bounds, unsigned long long *dtmin) {
    using R = EXG_R;
    if (c.np == 0) return;
    k_state_reduce<R><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.mat_dev, c.np, bounds, dtmin);
    EXG_CUDA_OK(cudaGetLastError());
}

template <class R, int ORD, bool TH>
static void p2g_cell_t(Ctx &c, int flags) {
    const int NCH = TH ? CH_ALL : CH_MOM_END;
    const int B3 = c.P.B * c.P.B * c.P.B;
    size_t sm = ((sizeof(SplineTables) + 15) & ~15) + sizeof(unsigned) * (fx_lo_words<R>() + 1) * NCH * B3;
    auto kern = k_p2g_cell<R, ORD, TH>;
    constexpr int nthr = P2GCfg<R, ORD, TH>::THREADS;
    EXG_CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    static int grid = 0;
    static size_t gsm = 0;
    if (!grid || gsm != sm) {
        int dev = 0, nsm = 0, per = 0;
        EXG_CUDA_OK(cudaGetDevice(&dev));
        EXG_CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        EXG_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, nthr, sm));
        grid = nsm * (per < 1 ? 1 : per);
        gsm = sm;
    }
    kern<<<grid, nthr, sm, c.stream>>>(c.P, c.A<R>(), c.sb.active, c.sb.tile_start, c.sb.cell_start, c.sb.perm,
                                       c.staging, c.ctl, flags);
    EXG_CUDA_OK(cudaGetLastError());
}

template <class R, int ORD, int V>
static void p2g_fact_v(Ctx &c) {
    const int B3 = c.P.B * c.P.B * c.P.B;
    size_t sm = ((sizeof(SplineTables) + 15) & ~15) + sizeof(unsigned) * (fx_lo_words<R>() + 1) * CH_MOM_END * B3;
    auto kern = k_p2g_fact<R, ORD, V>;
    constexpr int nthr = P2GVar<R, ORD, V>::THREADS;
    EXG_CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    static int grid = 0;
    static size_t gsm = 0;
    if (!grid || gsm != sm) {
        int dev = 0, nsm = 0, per = 0;
        EXG_CUDA_OK(cudaGetDevice(&dev));
        EXG_CUDA_OK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        EXG_CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, nthr, sm));
        grid = nsm * (per < 1 ? 1 : per);
        gsm = sm;
    }
    kern<<<grid, nthr, sm, c.stream>>>(c.P, c.A<R>(), c.sb.active, c.sb.tile_start, c.sb.cell_start, c.sb.perm,
                                       c.staging, c.ctl);
    EXG_CUDA_OK(cudaGetLastError());
}

template <class R, int ORD, bool TH>
static void p2g_t(Ctx &c, int flags) {
    if constexpr (P2GCfg<R, ORD, TH>::FACT) {
        switch (c.p2g_var) {
            case 1: p2g_fact_v<R, ORD, 1>(c); break;
            case 2: p2g_fact_v<R, ORD, 2>(c); break;
            default: p2g_fact_v<R, ORD, 0>(c); break;
        }
    } else {
        p2g_cell_t<R, ORD, TH>(c, flags);
    }
}

void EXG_SFX(launch_p2g)(Ctx &c, int flags) {
    using R = EXG_R;
    const bool th = (flags & (PF_TEMP | PF_SRC)) != 0;
    switch (c.P.uniform_order) {
        case 1: th ? p2g_t<R, 1, true>(c, flags) : p2g_t<R, 1, false>(c, flags); break;
        case 2: th ? p2g_t<R, 2, true>(c, flags) : p2g_t<R, 2, false>(c, flags); break;
        case 3: th ? p2g_t<R, 3, true>(c, flags) : p2g_t<R, 3, false>(c, flags); break;
        default: th ? p2g_t<R, 0, true>(c, flags) : p2g_t<R, 0, false>(c, flags); break;
    }
}

void EXG_SFX(launch_nodes)(Ctx &c, int mode, int flags, bool all_tiles) {
    using R = EXG_R;
    const bool th = (flags & (PF_TEMP | PF_SRC)) != 0;
    NodeBCArgs bc = make_bc(c);
    // walls only (no UDF wall tables, no level-set bodies, no temperature):
    // the lean instantiation, which inlines the wall BCs
    bool lean = !th && c.P.num_bodies == 0;
    for (int h = 0; h < 2; ++h)
        for (int d = 0; d < 3; ++d) lean = lean && bc.udf[h][d] == nullptr;
    static int pgrid = 0, pgrid_th = 0, pgrid_lean = 0;
    if (!pgrid) pgrid = persistent_grid(k_nodes<R, false>, 0);
    if (!pgrid_th) pgrid_th = persistent_grid(k_nodes<R, true>, 0);
    if (!pgrid_lean) pgrid_lean = persistent_grid(k_nodes<R, false, true>, 0);
    const int pg = th ? pgrid_th : (lean ? pgrid_lean : pgrid);  // the grid of the variant launched
    int grid = all_tiles ? (int)std::min<long long>(c.P.ntiles, pg) : pg;
    const int *tiles = all_tiles ? nullptr : c.sb.touched;
    if (th)
        k_nodes<R, true><<<grid, kThreads, 0, c.stream>>>(c.P, c.N<R>(), bc, tiles, c.sb.slot, c.staging, c.ctl, mode,
                                                          flags);
    else if (lean)
        k_nodes<R, false, true><<<grid, kThreads, 0, c.stream>>>(c.P, c.N<R>(), bc, tiles, c.sb.slot, c.staging,
                                                                 c.ctl, mode, flags);
    else
        k_nodes<R, false><<<grid, kThreads, 0, c.stream>>>(c.P, c.N<R>(), bc, tiles, c.sb.slot, c.staging, c.ctl,
                                                           mode, flags);
    EXG_CUDA_OK(cudaGetLastError());
}

template <class R, int ORD, bool LEAN, int V = 0>
static void g2p_lt(Ctx &c, int mode) {
    const int B3 = c.P.B * c.P.B * c.P.B;
    // tables, then one node block (two with TMA staging in FP32), each
    // 128-byte aligned
    const size_t tabb = (sizeof(SplineTables) + 127) & ~size_t(127);
    const size_t buf = (sizeof(R) * SmemNodes<R>::NS * B3 + 127) & ~size_t(127);
    const int nbuf = (c.tma && sizeof(R) == 4) ? 2 : 1;
    size_t sm = tabb + nbuf * buf + 128;  // + room to align the node blocks to 128 bytes
    auto kern = k_g2p_fused<R, ORD, LEAN, V>;
    constexpr int nthr = G2PVar<R, V>::THREADS;
    EXG_CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    static int grid = 0;
    static size_t gsm = 0;
    if (!grid || gsm != sm) {
        grid = persistent_grid(kern, sm, nthr);
        gsm = sm;
    }
    kern<<<grid, nthr, sm, c.stream>>>(c.P, c.A<R>(), c.Bp<R>(), c.N<R>(), make_bc(c), c.mat_dev, c.sb.active,
                                       c.sb.tile_start, c.sb.tile_count, c.sb.perm, c.sb.item_start, c.ctl, mode,
                                       c.tmap, c.tma ? 1 : 0, (long long)c.np);
    EXG_CUDA_OK(cudaGetLastError());
}
template <class R, int ORD>
static void g2p_t(Ctx &c, int mode) {
    if (g2p_lean(c)) {
        if constexpr (ORD == 2 || ORD == 3) {
            switch (c.g2p_var) {
                case 1: g2p_lt<R, ORD, true, 1>(c, mode); return;
                case 2: g2p_lt<R, ORD, true, 2>(c, mode); return;
                default: break;
            }
        }
        g2p_lt<R, ORD, true>(c, mode);
    } else {
        g2p_lt<R, ORD, false>(c, mode);
    }
}
void EXG_SFX(launch_g2p_fused)(Ctx &c, int mode) {
    using R = EXG_R;
    switch (c.P.uniform_order) {
        case 1: g2p_t<R, 1>(c, mode); break;
        case 2: g2p_t<R, 2>(c, mode); break;
        case 3: g2p_t<R, 3>(c, mode); break;
        default: g2p_t<R, 0>(c, mode); break;
    }
}

void EXG_SFX(launch_copy_lost)(Ctx &c) {
    if (c.np == 0) return;
    k_copy_lost<EXG_R><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.A<EXG_R>(), c.Bp<EXG_R>(), c.sb.key, c.np, c.ctl,
                                                                 c.specs.use_temp);
    EXG_CUDA_OK(cudaGetLastError());
}

void EXG_SFX(launch_g2p_simple)(Ctx &c, int uv, int us, double dt) {
    using R = EXG_R;
    if (c.np == 0) return;
    switch (c.P.uniform_order) {
        case 1: k_g2p_simple<R, 1><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, uv, us, dt); break;
        case 2: k_g2p_simple<R, 2><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, uv, us, dt); break;
        case 3: k_g2p_simple<R, 3><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, uv, us, dt); break;
        default: k_g2p_simple<R, 0><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, uv, us, dt); break;
    }
    EXG_CUDA_OK(cudaGetLastError());
}

void EXG_SFX(launch_fill_node)(Ctx &c, int comp, double value) {
    k_fill<EXG_R><<<nblocks(c.P.nnodes), kThreads, 0, c.stream>>>(c.N<EXG_R>().c[comp], c.P.nnodes, value);
    EXG_CUDA_OK(cudaGetLastError());
}

void EXG_SFX(launch_temp_node_op)(Ctx &c, int op, double dt) {
    k_temp_node_op<EXG_R><<<nblocks(c.P.nnodes), kThreads, 0, c.stream>>>(c.P, c.N<EXG_R>(), op, dt);
    EXG_CUDA_OK(cudaGetLastError());
}

void EXG_SFX(launch_temp_bcs)(Ctx &c, int walls, int udf, int ls, int dirichlet_only) {
    using R = EXG_R;
    const NodeBCArgs bc = make_bc(c);
    Nodes<R> &Nd = c.N<R>();
    if ((walls != TW_OFF || udf) && c.n_tface > 0) {
        k_temp_faces<R><<<nblocks(c.n_tface), kThreads, 0, c.stream>>>(c.P, Nd, bc, c.tface, c.n_tface, walls != TW_OFF,
                                                                       walls == TW_MASKED, udf, c.ctl);
        EXG_CUDA_OK(cudaGetLastError());
        k_temp_faces_store<R><<<nblocks(c.n_tface), kThreads, 0, c.stream>>>(c.P, Nd, c.tface, c.n_tface);
        EXG_CUDA_OK(cudaGetLastError());
    }
    if (!ls) return;
    for (int b = 0; b < c.P.num_bodies; ++b) {
        const int tb = c.P.body[b].temp_bc;
        if (!c.ls[b] || tb == 0 || (dirichlet_only && tb != 1)) continue;
        R *tmp = reinterpret_cast<R *>(c.ttmp);
        k_temp_levelset<R><<<nblocks(c.P.nnodes), kThreads, 0, c.stream>>>(c.P, Nd, c.ls[b], b,
                                                                           Nd.c[EXG_N_TEMPERATURE], tmp);
        EXG_CUDA_OK(cudaGetLastError());
        EXG_CUDA_OK(cudaMemcpyAsync(Nd.c[EXG_N_TEMPERATURE], tmp, sizeof(R) * c.P.nnodes, cudaMemcpyDeviceToDevice,
                                    c.stream));
    }
}

void EXG_SFX(launch_g2p_temp)(Ctx &c, int ut, int uq) {
    using R = EXG_R;
    if (c.np == 0) return;
    const int nb = nblocks(c.np);
    switch (c.P.uniform_order) {
        case 1: k_g2p_temp<R, 1><<<nb, kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, ut, uq); break;
        case 2: k_g2p_temp<R, 2><<<nb, kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, ut, uq); break;
        case 3: k_g2p_temp<R, 3><<<nb, kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, ut, uq); break;
        default: k_g2p_temp<R, 0><<<nb, kThreads, 0, c.stream>>>(c.P, c.A<R>(), c.N<R>(), c.np, ut, uq); break;
    }
    EXG_CUDA_OK(cudaGetLastError());
}

void EXG_SFX(launch_node_backup)(Ctx &c) {
    k_node_backup<EXG_R><<<nblocks(c.P.nnodes), kThreads, 0, c.stream>>>(c.P, c.N<EXG_R>());
    EXG_CUDA_OK(cudaGetLastError());
}
void EXG_SFX(launch_node_time_update)(Ctx &c, double dt) {
    k_node_time_update<EXG_R><<<nblocks(c.P.nnodes), kThreads, 0, c.stream>>>(c.P, c.N<EXG_R>(), dt);
    EXG_CUDA_OK(cudaGetLastError());
}
void EXG_SFX(launch_node_bcs)(Ctx &c) {
    k_node_bcs<EXG_R><<<nblocks(c.P.nnodes), kThreads, 0, c.stream>>>(c.P, c.N<EXG_R>(), make_bc(c), c.ctl);
    EXG_CUDA_OK(cudaGetLastError());
}
void EXG_SFX(launch_move)(Ctx &c, double dt) {
    if (c.np == 0) return;
    k_move<EXG_R><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, c.A<EXG_R>(), make_bc(c), c.np, dt, c.ctl);
    EXG_CUDA_OK(cudaGetLastError());
}
void EXG_SFX(launch_volume)(Ctx &c) {
    if (c.np == 0) return;
    k_vol_stress<EXG_R><<<nblocks(c.np), kThreads, 0, c.stream>>>(c.P, c.A<EXG_R>(), c.mat_dev, c.np, 0.0, 0.0, 1, 0);
    EXG_CUDA_OK(cudaGetLastError());
}
void EXG_SFX(launch_stress)(Ctx &c, double time, double dt, bool total) {
    if (c.np == 0) return;
    double asr = (time < c.P.applied_sr_time) ? c.P.applied_sr : 0.0;
    Params P = c.P;
    if (total) P.delta_strain = 0;  // Initialise_Internal_Forces: total formulation
    k_vol_stress<EXG_R><<<nblocks(c.np), kThreads, 0, c.stream>>>(P, c.A<EXG_R>(), c.mat_dev, c.np, dt, asr, 0, 1);
    EXG_CUDA_OK(cudaGetLastError());
}
void EXG_SFX(launch_diag)(Ctx &c, double *out_dev) {
    int nb = nblocks(c.np > 0 ? c.np : 1);
    double *part = out_dev + 32;
    k_diag_partial<EXG_R><<<nb, kThreads, 0, c.stream>>>(c.P, c.A<EXG_R>(), c.np, part);
    k_diag_final<<<1, 32, 0, c.stream>>>(part, nb, out_dev);
    EXG_CUDA_OK(cudaGetLastError());
}

// ---- host transfers of particle fields (through the device staging buffer)
void EXG_SFX(h2d_field)(Ctx &c, void *dst, const double *host, long long n, double sub) {
    using R = EXG_R;
    if (n == 0) return;
    if (sizeof(R) == 8 && sub == 0.0) {
        EXG_CUDA_OK(cudaMemcpyAsync(dst, host, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
        return;
    }
    EXG_CUDA_OK(cudaMemcpyAsync(c.stage, host, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
    k_from_f64<R><<<nblocks(n), kThreads, 0, c.stream>>>(c.stage, reinterpret_cast<R *>(dst), n, sub);
    EXG_CUDA_OK(cudaGetLastError());
}
void EXG_SFX(d2h_field)(Ctx &c, const void *src, const int32_t *pid, double *host, long long n, double add) {
    using R = EXG_R;
    if (n == 0) return;
    k_to_f64_unperm<R><<<nblocks(n), kThreads, 0, c.stream>>>(reinterpret_cast<const R *>(src), pid, c.stage, n, add);
    EXG_CUDA_OK(cudaGetLastError());
    EXG_CUDA_OK(cudaMemcpyAsync(host, c.stage, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream));
}
#if defined(EXG_R_FP64)
void d2h_positions(Ctx &c, double *const x[3], const int32_t *pid, double *host, long long n) {
    for (int d = 0; d < 3; ++d) {
        k_to_f64_unperm<double><<<nblocks(n), kThreads, 0, c.stream>>>(x[d], pid, c.stage, n, 0.0);
        EXG_CUDA_OK(cudaGetLastError());
        EXG_CUDA_OK(cudaMemcpyAsync(host + (size_t)d * n, c.stage, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                    c.stream));
    }
}
void d2h_int(Ctx &c, const void *src, int bytes, const int32_t *pid, int32_t *host, long long n) {
    int32_t *st = reinterpret_cast<int32_t *>(c.stage);
    if (bytes == 1)
        k_unperm_i32<uint8_t><<<nblocks(n), kThreads, 0, c.stream>>>(reinterpret_cast<const uint8_t *>(src), pid, st, n);
    else
        k_unperm_i32<int32_t><<<nblocks(n), kThreads, 0, c.stream>>>(reinterpret_cast<const int32_t *>(src), pid, st, n);
    EXG_CUDA_OK(cudaGetLastError());
    EXG_CUDA_OK(cudaMemcpyAsync(host, st, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, c.stream));
}
#endif

// ---- batched scenes
template <class R>
static bool batch_descriptors_t(Batch &b) {
    const size_t n = b.scenes.size();
    bool changed = false;
    for (int par = 0; par < 2; ++par) {
        std::vector<SceneDesc<R>> d(n);
        for (size_t s = 0; s < n; ++s) {
            Ctx &c = *b.scenes[s];
            SceneDesc<R> &x = d[s];
            std::memset(&x, 0, sizeof(x));
            x.P = c.P;
            // at the batch's current parity the scene reads its current
            // storage and writes the other one; the next parity swaps them
            const bool now = (par == b.parity);
            x.A = now ? c.A<R>() : c.Bp<R>();
            x.Bo = now ? c.Bp<R>() : c.A<R>();
            x.N = c.N<R>();
            x.bc = make_bc(c);
            x.mats = c.mat_dev;
            x.active = c.sb.active;
            x.start = c.sb.tile_start;
            x.count = c.sb.tile_count;
            x.cell_start = c.sb.cell_start;
            x.touched = c.sb.touched;
            x.slot = c.sb.slot;
            x.perm = c.sb.perm;
            x.staging = c.staging;
            x.ctl = c.ctl;
        }
        const unsigned char *raw = reinterpret_cast<const unsigned char *>(d.data());
        std::vector<unsigned char> h(raw, raw + n * sizeof(SceneDesc<R>));
        if (h != b.desc_host[par]) {
            changed = true;
            if (!b.desc[par]) EXG_CUDA_OK(cudaMalloc(&b.desc[par], h.size()));
            EXG_CUDA_OK(cudaMemcpy(b.desc[par], h.data(), h.size(), cudaMemcpyHostToDevice));
            b.desc_host[par] = std::move(h);
        }
        // the batched sort's view of the same scenes
        std::vector<SortDesc> sd(n);
        for (size_t s = 0; s < n; ++s) {
            Ctx &c = *b.scenes[s];
            SortDesc &x = sd[s];
            std::memset(&x, 0, sizeof(x));
            x.P = c.P;
            const Parts<R> &A = (par == b.parity) ? c.A<R>() : c.Bp<R>();
            for (int k = 0; k < 3; ++k) x.x[k] = A.x[k];
            x.np = c.np;
            x.cap = (int)c.cap;
            x.key = c.sb.key;
            x.tile_count = c.sb.tile_count;
            x.tile_fill = c.sb.tile_fill;
            x.tile_start = c.sb.tile_start;
            x.active = c.sb.active;
            x.slot = c.sb.slot;
            x.item_start = c.sb.item_start;
            x.touched = c.sb.touched;
            x.cell_start = c.sb.cell_start;
            x.touched_step = c.sb.touched_step;
            x.bucket = c.sb.bucket;
            x.perm = c.sb.perm;
            x.ctl = c.ctl;
            x.bounds_cur = c.bounds_cur;
        }
        const unsigned char *sraw = reinterpret_cast<const unsigned char *>(sd.data());
        std::vector<unsigned char> sh(sraw, sraw + n * sizeof(SortDesc));
        if (sh != b.sdesc_host[par]) {
            changed = true;
            if (!b.sdesc[par]) EXG_CUDA_OK(cudaMalloc(&b.sdesc[par], sh.size()));
            EXG_CUDA_OK(cudaMemcpy(b.sdesc[par], sh.data(), sh.size(), cudaMemcpyHostToDevice));
            b.sdesc_host[par] = std::move(sh);
        }
    }
    // block and tile prefix sums of the batched per-particle and per-tile
    // kernels (particle counts change only with an upload)
    std::vector<int> pre_blocks(n + 1, 0), pre_tiles(n + 1, 0);
    for (size_t s = 0; s < n; ++s) {
        const Ctx &c = *b.scenes[s];
        pre_blocks[s + 1] = pre_blocks[s] + (int)((c.np + kBatchThreads - 1) / kBatchThreads);
        pre_tiles[s + 1] = pre_tiles[s] + (int)c.P.ntiles;
    }
    if (changed || pre_blocks[n] != b.total_blocks || pre_tiles[n] != b.total_tiles) {
        EXG_CUDA_OK(cudaMemcpy(b.bctl->pre_blocks, pre_blocks.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        EXG_CUDA_OK(cudaMemcpy(b.bctl->pre_tiles, pre_tiles.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
        b.total_blocks = pre_blocks[n];
        b.total_tiles = pre_tiles[n];
        changed = true;
    }
    b.desc_bytes = sizeof(SceneDesc<R>);
    return changed;
}
bool EXG_SFX(batch_descriptors)(Batch &b) { return batch_descriptors_t<EXG_R>(b); }

template <class R, int ORD, bool LEAN>
static void batch_g2p_t(Batch &b, const SceneDesc<R> *d, int B3) {
    const size_t sm = ((sizeof(SplineTables) + 15) & ~15) + sizeof(R) * SmemNodes<R>::NS * B3;
    auto kern = k_g2p_batch<R, ORD, LEAN>;
    EXG_CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    static int grid = 0;
    static size_t gsm = 0;
    if (!grid || gsm != sm) {
        grid = persistent_grid(kern, sm, EXG_G2P_THREADS);
        gsm = sm;
    }
    kern<<<grid, EXG_G2P_THREADS, sm, b.stream>>>(d, b.bctl, GM_FULL);
    EXG_CUDA_OK(cudaGetLastError());
}

template <class R, int ORD>
static void batch_p2g_t(Batch &b) {
    Ctx &c0 = *b.scenes[0];
    const SceneDesc<R> *d = reinterpret_cast<const SceneDesc<R> *>(b.desc[b.parity]);
    const int B3 = c0.P.B * c0.P.B * c0.P.B;
    constexpr int NCH = CH_MOM_END;
    const size_t sm = ((sizeof(SplineTables) + 15) & ~15) + sizeof(unsigned) * (fx_lo_words<R>() + 1) * NCH * B3;
    auto kern = k_p2g_batch<R, ORD, false>;
    constexpr int nthr = P2GCfg<R, ORD, false>::THREADS;
    EXG_CUDA_OK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    static int grid = 0;
    static size_t gsm = 0;
    if (!grid || gsm != sm) {
        grid = persistent_grid(kern, sm, nthr);
        gsm = sm;
    }
    kern<<<grid, nthr, sm, b.stream>>>(d, b.bctl, B3);
    EXG_CUDA_OK(cudaGetLastError());
}
template <class R>
static void batch_nodes_t(Batch &b) {
    const SceneDesc<R> *d = reinterpret_cast<const SceneDesc<R> *>(b.desc[b.parity]);
    static int grid = 0;
    if (!grid) grid = persistent_grid(k_nodes_batch<R, false>, 0);
    k_nodes_batch<R, false><<<grid, kThreads, 0, b.stream>>>(d, b.bctl, NM_FUSED, PF_MASS | PF_VEL | PF_FORCE);
    EXG_CUDA_OK(cudaGetLastError());
}
template <class R, int ORD>
static void batch_g2p_o(Batch &b) {
    Ctx &c0 = *b.scenes[0];
    const SceneDesc<R> *d = reinterpret_cast<const SceneDesc<R> *>(b.desc[b.parity]);
    const int B3 = c0.P.B * c0.P.B * c0.P.B;
    bool lean = true;
    for (Ctx *s : b.scenes) lean = lean && g2p_lean(*s);
    if (lean)
        batch_g2p_t<R, ORD, true>(b, d, B3);
    else
        batch_g2p_t<R, ORD, false>(b, d, B3);
}
void EXG_SFX(launch_batch_p2g)(Batch &b) {
    using R = EXG_R;
    switch (b.scenes[0]->P.uniform_order) {
        case 1: batch_p2g_t<R, 1>(b); break;
        case 2: batch_p2g_t<R, 2>(b); break;
        case 3: batch_p2g_t<R, 3>(b); break;
        default: batch_p2g_t<R, 0>(b); break;
    }
}
void EXG_SFX(launch_batch_nodes)(Batch &b) { batch_nodes_t<EXG_R>(b); }
void EXG_SFX(launch_batch_g2p)(Batch &b) {
    using R = EXG_R;
    switch (b.scenes[0]->P.uniform_order) {
        case 1: batch_g2p_o<R, 1>(b); break;
        case 2: batch_g2p_o<R, 2>(b); break;
        case 3: batch_g2p_o<R, 3>(b); break;
        default: batch_g2p_o<R, 0>(b); break;
    }
}
void EXG_SFX(launch_batch_core)(Batch &b) {
    EXG_SFX(launch_batch_p2g)(b);
    EXG_SFX(launch_batch_nodes)(b);
    EXG_SFX(launch_batch_g2p)(b);
}
void EXG_SFX(launch_batch_finish)(Batch &b) {
    using R = EXG_R;
    const SceneDesc<R> *dr = reinterpret_cast<const SceneDesc<R> *>(b.desc[b.parity]);
    if (b.total_blocks > 0)
        k_bb_copy_lost<R><<<b.total_blocks, kBatchThreads, 0, b.stream>>>(dr, b.sdesc[b.parity], b.bctl,
                                                                          b.scenes[0]->specs.use_temp);
    const int ns = (int)b.scenes.size();
    k_bb_time_advance<<<nblocks(ns), kThreads, 0, b.stream>>>(b.sdesc[b.parity], ns);
    EXG_CUDA_OK(cudaGetLastError());
}

#if defined(EXG_R_FP64)
void launch_batch_plan(Batch &b) {
    k_batch_plan<<<1, kThreads, 0, b.stream>>>(b.bctl, b.ctls);
    EXG_CUDA_OK(cudaGetLastError());
}

void launch_batch_sort(Batch &b) {
    const SortDesc *d = b.sdesc[b.parity];
    const int ns = (int)b.scenes.size();
    const Ctx &c0 = *b.scenes[0];
    k_bb_start<<<nblocks(std::max(b.total_tiles, ns)), kThreads, 0, b.stream>>>(d, b.bctl);
    if (b.total_blocks > 0) k_bb_keys<<<b.total_blocks, kBatchThreads, 0, b.stream>>>(d, b.bctl);
    k_bb_tile_scan<<<ns, 1024, 0, b.stream>>>(d);
    if (b.total_blocks > 0) k_bb_scatter<<<b.total_blocks, kBatchThreads, 0, b.stream>>>(d, b.bctl);
    // active-tile prefix sums for the batched tile sort
    k_batch_plan<<<1, kThreads, 0, b.stream>>>(b.bctl, b.ctls);
    const int ncell = c0.P.T * c0.P.T * c0.P.T;
    const size_t sm = sizeof(int) * (3 * ncell + kSortCap);
    EXG_CUDA_OK(cudaFuncSetAttribute(k_bb_tile_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    static int sgrid = 0;
    if (!sgrid) sgrid = persistent_grid(k_bb_tile_sort, sm);
    k_bb_tile_sort<<<sgrid, kThreads, sm, b.stream>>>(d, b.bctl, ncell);
    k_bb_touched<<<nblocks(b.total_tiles), kThreads, 0, b.stream>>>(d, b.bctl);
    const int W = (c0.P.uniform_order == 1) ? 2 : (c0.P.dual ? 3 : 4);
    k_bb_scales<<<ns, 32, 0, b.stream>>>(d, W * W * W, c0.precision == EXG_PREC_FP64 ? kFxBits64 : kFxBits32);
    EXG_CUDA_OK(cudaGetLastError());
}
#endif


#if defined(EXG_R_FP64)
// ====================================================================== no-alloc P2G
// exg_p2g_momentum_noalloc: P2G of mass, momentum and force for callers that
// must not allocate device memory (see include/exg.h).  Its scratch -- the
// 64-bit fixed-point node sums, the per-channel bounds and scales -- lives in
// this file-scope device array instead of cudaMalloc'd buffers.  Every GPU
// that loads the library holds the array until the process exits.
namespace {
constexpr long long kNaNodes = EXG_NOALLOC_MAX_NODES;
constexpr int kNaCh = CH_MOM_END;  // mass, momentum(3), force(3)
// [kNaCh * kNaNodes] node sums, then 17 header words -- 7 bound words and a
// flag word (set when an input term is not finite), 8 scale words, one word
// for the largest particle count of a cell -- then kNaNodes 32-bit cell counts
constexpr long long kNaWords = kNaCh * kNaNodes + 17 + kNaNodes / 2;
constexpr int kNaFlagWord = 7;  // header word after the kNaCh bound words
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNaWords];

struct NaArgs {
    const double *pos;
    const double *rdata;
    const int32_t *idata;
    long long np;
    double *mass, *vel, *frc;
    unsigned long long *acc;  // device address of g_noalloc_scratch
};

// Zeroes the words this call uses: each channel's first nnodes sums, the 17
// header words and the count words of the grid's cells (the rest of the
// array keeps whatever an earlier, larger grid left there and is not read).
__global__ void k_na_clear(Params P, unsigned long long *acc) {
    const long long ncells = (long long)P.nc[0] * P.nc[1] * P.nc[2];
    const long long nsum = kNaCh * P.nnodes, ncnt = (ncells + 1) / 2;
    const long long n = nsum + 17 + ncnt;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        long long w;
        if (i < nsum)
            w = (i / P.nnodes) * kNaNodes + i % P.nnodes;
        else
            w = kNaCh * kNaNodes + (i - nsum);
        acc[w] = 0ull;
    }
}

// particles per cell, and the largest count (the fixed-point range bound
// uses it as the context path uses the sort's maximum)
__global__ void k_na_count(Params P, NaArgs a) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= a.np || a.idata[(long long)EXG_I_PHASE * a.np + p] != 0) return;
    const double x[3] = {a.pos[p], a.pos[a.np + p], a.pos[2 * a.np + p]};
    int iv[3];
    cell_of(P, x, iv);
    if (iv[0] < 0 || iv[0] >= P.nc[0] || iv[1] < 0 || iv[1] >= P.nc[1] || iv[2] < 0 || iv[2] >= P.nc[2]) return;
    unsigned *cnt = reinterpret_cast<unsigned *>(a.acc + kNaCh * kNaNodes + 17);
    const unsigned old = atomicAdd(&cnt[((long long)iv[2] * P.nc[1] + iv[1]) * P.nc[0] + iv[0]], 1u);
    atomicMax(a.acc + kNaCh * kNaNodes + 16, (unsigned long long)(old + 1u));
}

// per-channel largest |term| (as ordered bits) over phase-0 particles
__global__ void k_na_bounds(Params P, NaArgs a) {
    long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= a.np || a.idata[(long long)EXG_I_PHASE * a.np + p] != 0) return;
    auto R = [&](int f) { return a.rdata[(long long)f * a.np + p]; };
    unsigned long long *bnd = a.acc + kNaCh * kNaNodes;
    const double m = R(EXG_R_MASS), vol = R(EXG_R_VOLUME);
    double b[kNaCh];
    b[CH_M] = fabs(m);
    const int rowi[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    for (int d = 0; d < 3; ++d) {
        b[CH_P + d] = fabs(m * R(EXG_R_VEL + d));
        double s = 0.0;
        for (int j = 0; j < 3; ++j) s += fabs(R(EXG_R_STRESS + rowi[d][j])) * 2.0 * P.dxi[j];
        b[CH_F + d] = fabs(m * P.gravity[d]) + (P.external_loads ? fabs(P.extforce[d]) : 0.0) + fabs(vol) * s;
    }
    for (int c = 0; c < kNaCh; ++c) atomicMax(&bnd[c], dbits(b[c]));
}

// scale 2^e per channel so that (particles per cell) x (stencil cells) x
// (largest term) x 2 < 2^61, the bound of the context path's FP64 k_scales
__global__ void k_na_scale(NaArgs a, int stencil_cells) {
    const int c = threadIdx.x;
    if (c >= kNaCh) return;
    unsigned long long *bnd = a.acc + kNaCh * kNaNodes;
    const unsigned long long ppc = bnd[16];
    const double S = bitsd(bnd[c]) * (double)(ppc > 0 ? ppc : 1) * (double)stencil_cells * 2.0;
    double sc = 1.0;
    if (S > 0.0 && S < 1e300) {
        int ex;
        frexp(S, &ex);
        sc = ldexp(1.0, max(-100, min(100, 61 - ex)));
    } else if (!(S >= 0.0) || S >= 1e300) {
        // a non-finite (or absurdly large) input term: no fixed-point scale
        // can hold it, so k_na_finish writes NaN to every output
        atomicOr(&bnd[kNaFlagWord], 1ull);
    }
    bnd[8 + c] = dbits(sc);
}

template <int ORD>
__global__ void __launch_bounds__(kThreads) k_na_deposit(Params P, NaArgs a) {
    constexpr int W = Stc<ORD>::W, LO = Stc<ORD>::LO;
    __shared__ SplineTables tab;
    load_tables(&tab);
    __syncthreads();
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= a.np || a.idata[(long long)EXG_I_PHASE * a.np + p] != 0) return;
    auto R = [&](int f) { return a.rdata[(long long)f * a.np + p]; };
    const unsigned long long *bnd = a.acc + kNaCh * kNaNodes;
    double sc[kNaCh];
    for (int c = 0; c < kNaCh; ++c) sc[c] = bitsd(bnd[8 + c]);
    const double x[3] = {a.pos[p], a.pos[a.np + p], a.pos[2 * a.np + p]};
    int iv[3];
    cell_of(P, x, iv);
    if (iv[0] < 0 || iv[0] >= P.nc[0] || iv[1] < 0 || iv[1] >= P.nc[1] || iv[2] < 0 || iv[2] >= P.nc[2]) return;
    AxisW<double, W> ax, ay, az;
    axis_weights<double, W, LO>(tab, P, 0, x[0], iv[0], ax);
    axis_weights<double, W, LO>(tab, P, 1, x[1], iv[1], ay);
    axis_weights<double, W, LO>(tab, P, 2, x[2], iv[2], az);
    const double m = R(EXG_R_MASS), vol = R(EXG_R_VOLUME);
    double mv[3], s[6];
    for (int d = 0; d < 3; ++d) mv[d] = m * R(EXG_R_VEL + d);
    for (int c = 0; c < 6; ++c) s[c] = R(EXG_R_STRESS + c);
    const bool slab = P.external_loads && x[0] > P.slab_lo[0] && x[0] < P.slab_hi[0] && x[1] > P.slab_lo[1] &&
                      x[1] < P.slab_hi[1] && x[2] > P.slab_lo[2] && x[2] < P.slab_hi[2];
    for (int sz = 0; sz < W; ++sz)
        for (int sy = 0; sy < W; ++sy)
            for (int sx = 0; sx < W; ++sx) {
                const double wx = ax.w[sx], wy = ay.w[sy], wz = az.w[sz];
                const double dx = ax.dw[sx], dy = ay.dw[sy], dz = az.dw[sz];
                if ((wx == 0.0 && dx == 0.0) || (wy == 0.0 && dy == 0.0) || (wz == 0.0 && dz == 0.0)) continue;
                const long long ni = node_index(P, iv[0] + LO + sx, iv[1] + LO + sy, iv[2] + LO + sz);
                if (ni < 0) continue;
                const double N = wx * wy * wz;
                const double g[3] = {dx * wy * wz, wx * dy * wz, wx * wy * dz};
                double v[kNaCh];
                v[CH_M] = m * N;
                for (int d = 0; d < 3; ++d) {
                    v[CH_P + d] = mv[d] * N;
                    const double tv = s[d == 0 ? 0 : (d == 1 ? 1 : 2)] * g[0] +
                                      s[d == 0 ? 1 : (d == 1 ? 3 : 4)] * g[1] + s[d == 0 ? 2 : (d == 1 ? 4 : 5)] * g[2];
                    v[CH_F + d] = (m * P.gravity[d] * N + (slab ? P.extforce[d] * N : 0.0)) + (-vol * tv);
                }
                for (int c = 0; c < kNaCh; ++c) {
                    const long long q = __double2ll_rn(v[c] * sc[c]);
                    if (q) atomicAdd(&a.acc[(long long)c * kNaNodes + ni], (unsigned long long)q);
                }
            }
}

// node sums -> the caller's arrays: mass, velocity p/m (m >= mass_tolerance,
// as deposit_onto_grid_momentum normalises, mpm_particle_grid_ops.cpp:602-615),
// force
__global__ void k_na_finish(Params P, NaArgs a) {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= P.nnodes) return;
    const unsigned long long *bnd = a.acc + kNaCh * kNaNodes;
    // periodic axes: node ncells reads node 0
    int id[3] = {(int)(n % P.nn[0]), (int)((n / P.nn[0]) % P.nn[1]), (int)(n / ((long long)P.nn[0] * P.nn[1]))};
    const long long src = node_index(P, id[0], id[1], id[2]);
    double v[kNaCh];
    const bool bad = bnd[kNaFlagWord] != 0ull;
    for (int c = 0; c < kNaCh; ++c)
        v[c] = bad ? __longlong_as_double(0x7ff8000000000000ll)
                   : (double)(long long)a.acc[(long long)c * kNaNodes + src] * (1.0 / bitsd(bnd[8 + c]));
    const double m = v[CH_M];
    a.mass[n] = m;
    for (int d = 0; d < 3; ++d) {
        double vel = v[CH_P + d];
        if (m > 0.0) vel = (m >= P.mass_tol) ? v[CH_P + d] / m : 0.0;
        a.vel[(long long)d * P.nnodes + n] = vel;
        a.frc[(long long)d * P.nnodes + n] = v[CH_F + d];
    }
}

// per device: the scratch array's device address, set once under its flag
constexpr int kNaMaxDevices = 64;
std::once_flag g_na_once[kNaMaxDevices];
std::atomic<unsigned long long *> g_na_addr[kNaMaxDevices];
}  // namespace

// Builds the kernel parameters of a specs (also used by the context).
void build_params_for(const exg_specs &s, Params &P);

int noalloc_p2g(const exg_specs *specs, const exg_particle_soa *dev, double *mass, double *vel, double *frc,
                cudaStream_t stream, std::string &err) {
    Params P;
    build_params_for(*specs, P);
    if (P.nnodes > kNaNodes) {
        err = "exg_p2g_momentum_noalloc: the grid has " + std::to_string(P.nnodes) +
              " nodes; this entry point's static scratch holds at most " + std::to_string(kNaNodes) +
              " (EXG_NOALLOC_MAX_NODES)";
        return EXG_ERR_OVERFLOW;
    }
    int dev_id = 0;
    if (cudaGetDevice(&dev_id) != cudaSuccess || dev_id < 0 || dev_id >= kNaMaxDevices) {
        err = "exg_p2g_momentum_noalloc: no current CUDA device";
        return EXG_ERR_CUDA;
    }
    // one-time set-up on this device (outside any stream capture): the
    // device address of the scratch array and the spline tables.  A failed
    // set-up throws out of call_once, which leaves the flag unset, so the
    // next call retries it.
    try {
        std::call_once(g_na_once[dev_id], [dev_id] {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                throw std::runtime_error(std::string("exg_p2g_momentum_noalloc: cudaGetSymbolAddress failed: ") +
                                         cudaGetErrorString(e));
            upload_tables_fp64();
            g_na_addr[dev_id].store(reinterpret_cast<unsigned long long *>(ptr), std::memory_order_release);
        });
    } catch (const std::exception &ex) {
        err = ex.what();
        return EXG_ERR_CUDA;
    }
    NaArgs a;
    a.pos = dev->pos;
    a.rdata = dev->rdata;
    a.idata = dev->idata;
    a.np = dev->np;
    a.mass = mass;
    a.vel = vel;
    a.frc = frc;
    a.acc = g_na_addr[dev_id].load(std::memory_order_acquire);
    {
        const long long ncells = (long long)P.nc[0] * P.nc[1] * P.nc[2];
        const long long nclear = kNaCh * P.nnodes + 17 + (ncells + 1) / 2;
        k_na_clear<<<std::min(nblocks(nclear), 4096), kThreads, 0, stream>>>(P, a.acc);
    }
    if (a.np > 0) {
        k_na_bounds<<<nblocks(a.np), kThreads, 0, stream>>>(P, a);
        k_na_count<<<nblocks(a.np), kThreads, 0, stream>>>(P, a);
    }
    const int W = (P.uniform_order == 1) ? 2 : 4;
    k_na_scale<<<1, 32, 0, stream>>>(a, W * W * W);
    if (a.np > 0) {
        switch (P.uniform_order) {
            case 1: k_na_deposit<1><<<nblocks(a.np), kThreads, 0, stream>>>(P, a); break;
            case 2: k_na_deposit<2><<<nblocks(a.np), kThreads, 0, stream>>>(P, a); break;
            case 3: k_na_deposit<3><<<nblocks(a.np), kThreads, 0, stream>>>(P, a); break;
            default: k_na_deposit<0><<<nblocks(a.np), kThreads, 0, stream>>>(P, a); break;
        }
    }
    k_na_finish<<<nblocks(P.nnodes), kThreads, 0, stream>>>(P, a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("exg_p2g_momentum_noalloc: ") + cudaGetErrorString(e);
        return EXG_ERR_CUDA;
    }
    return EXG_OK;
}
#endif  // EXG_R_FP64

}  // namespace exg
