// The deterministic space-charge deposit: contributions (records) sorted by cell with a
// stable LSD radix sort, summed per cell by warp segmented reductions in record order, and
// added to the nodes by a gather in a fixed order.  No floating-point atomics: every call
// on the same records gives the same node charges bit for bit.
//
// The per-record shape is the reference's area weighting
// (kernels/deposit_trajectories_2d/deposit_trajectories_2d_pyccel.py:28-59,
//  kernels/trace_trajectories_2d/trace_trajectories_2d_pyccel.py:397-423): a charge q at
// (u, w) in cell c adds (1-u)(1-w)q, (1-u)w q, u(1-w)q and u w q to the nodes c, c+1,
// c+ny, c+ny+1; a record holds those four charges (the sums of a run of a trajectory's
// steps in one cell, from the tracer), and its key the cell, or the sentinel for none.

#include "common.cuh"

namespace bt {

namespace {

constexpr int kThreads = 256;  // = the radix (one thread per digit in the scans)
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;
constexpr int kRadix = 256;      // 8-bit digits
constexpr int kRadixMax = 1024;  // up to 10-bit digits, when they save a pass
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;

// The record count of a sort or reduction: `n` from the host, or, where the caller gives
// one, the count the device holds (at most n; the grids are sized for n).
__device__ __forceinline__ i64 record_count(i64 n, const i64 *n_dev) { return n_dev ? *n_dev : n; }

// Keys equal to `skip` (a sort's first pass: the records with no charge) are left out of
// the counts and the output; kNoSkip leaves none out.
constexpr uint32_t kNoSkip = 0xffffffffu;

template <int R>
__global__ void radix_hist(const uint32_t *__restrict__ keys, i64 n_host,
                           const i64 *__restrict__ n_dev, uint32_t skip, int shift,
                           uint32_t *__restrict__ hist, int nblocks) {
    __shared__ uint32_t h[R];
    const i64 n = record_count(n_host, n_dev);
    for (int d = threadIdx.x; d < R; d += kThreads) h[d] = 0;
    __syncthreads();
    const i64 base = (i64)blockIdx.x * kTile;
    uint32_t key[kItems];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {  // the loads first, all in flight
        const i64 r = base + (i64)i * kThreads + threadIdx.x;
        key[i] = r < n ? keys[r] : skip;
    }
#pragma unroll
    for (int i = 0; i < kItems; ++i)
        if (key[i] != skip) atomicAdd(&h[(key[i] >> shift) & (R - 1)], 1u);
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kThreads) hist[(i64)d * nblocks + blockIdx.x] = h[d];
}

// Inclusive scan of one value per thread over a block of kThreads threads.
__device__ uint32_t block_inclusive_scan(uint32_t v, uint32_t *warp_sums) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, v, off);
        if (lane >= off) v += y;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < kWarps ? warp_sums[lane] : 0;
#pragma unroll
        for (int off = 1; off < kWarps; off <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, s, off);
            if (lane >= off) s += y;
        }
        if (lane < kWarps) warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t out = v + (warp > 0 ? warp_sums[warp - 1] : 0);
    __syncthreads();
    return out;
}

// Row d of hist (one digit over all blocks) to its exclusive prefix; the row total.
__global__ void radix_row_scan(const uint32_t *__restrict__ hist, uint32_t *__restrict__ offs,
                               uint32_t *__restrict__ totals, int nblocks) {
    __shared__ uint32_t warp_sums[kWarps];
    __shared__ uint32_t carry;
    const i64 row = (i64)blockIdx.x * nblocks;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int start = 0; start < nblocks; start += kThreads) {
        const int b = start + threadIdx.x;
        const uint32_t v = b < nblocks ? hist[row + b] : 0;
        const uint32_t incl = block_inclusive_scan(v, warp_sums);
        const uint32_t c = carry;
        if (b < nblocks) offs[row + b] = c + incl - v;
        __syncthreads();
        if (threadIdx.x == kThreads - 1) carry = c + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// Exclusive prefix of the R digit totals; thread t scans digits t * R / kThreads onwards.
// `count`, when not NULL, gets the number of records the pass sorts.
template <int R>
__global__ void radix_digit_base(const uint32_t *__restrict__ totals, uint32_t *__restrict__ base,
                                 i64 *__restrict__ count) {
    __shared__ uint32_t warp_sums[kWarps];
    constexpr int D = R / kThreads;
    uint32_t mine[D];
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        mine[k] = totals[threadIdx.x * D + k];
        v += mine[k];
    }
    const uint32_t inclusive = block_inclusive_scan(v, warp_sums);
    uint32_t run = inclusive - v;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        base[threadIdx.x * D + k] = run;
        run += mine[k];
    }
    if (count && threadIdx.x == kThreads - 1) *count = inclusive;
}

// Stable scatter of one tile of kTile records.  Warp w ranks the tile's items
// [w * kTile / kWarps, (w + 1) * kTile / kWarps) in order, 32 at a time (peers of a digit
// by __match_any_sync, a running count per warp and digit in shared memory: no block
// barrier in the loop); the counts are then turned into per-warp offsets in warp order and
// the tile's digit starts, the tile is sorted by digit in shared memory, and written out in
// order, so that the records of one digit go to consecutive addresses (coalesced runs).
// The shared array first holds the counts, then the sorted tile.
template <int R>
__global__ void __launch_bounds__(kThreads) radix_scatter(
    const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in, i64 n_host,
    const i64 *__restrict__ n_dev, uint32_t skip, int shift, const uint32_t *__restrict__ offs,
    const uint32_t *__restrict__ base, int nblocks, uint32_t *__restrict__ keys_out,
    uint32_t *__restrict__ vals_out) {
    static_assert(kWarps * R * 4 <= kTile * 8, "the counts must fit the tile's space");
    constexpr int D = R / kThreads;             // digits a thread scans
    constexpr int kPerWarp = kTile / kWarps;    // items a warp ranks
    __shared__ __align__(16) uint32_t space[2 * kTile];  // counts [kWarps][R], then the tile
    __shared__ uint32_t start[R];               // the tile's first slot of each digit
    __shared__ uint32_t run[R];                 // the digit's first global slot for this tile
    __shared__ uint32_t warp_sums[kWarps];
    __shared__ uint32_t tile_count;             // the tile's records that are sorted
    uint32_t *count = space;
    const i64 n = record_count(n_host, n_dev);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int d = t; d < kWarps * R; d += kThreads) count[d] = 0;
    __syncthreads();
    const i64 tile = (i64)blockIdx.x * kTile;
    const unsigned below = (1u << lane) - 1u;
    uint32_t key[kItems], val[kItems], pos[kItems];
    unsigned valid_mask = 0;  // bit i: item i is sorted
    // every load of the tile first (all in flight at once), then the ranking
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const i64 r = tile + (i64)warp * kPerWarp + (i64)i * 32 + lane;
        key[i] = r < n ? keys_in[r] : skip;
        val[i] = r < n ? (vals_in ? vals_in[r] : (uint32_t)r) : 0u;
    }
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const i64 r = tile + (i64)warp * kPerWarp + (i64)i * 32 + lane;
        const bool valid = r < n && key[i] != skip;
        if (valid) valid_mask |= 1u << i;
        if (!valid) val[i] = 0u;
        const uint32_t d = (key[i] >> shift) & (R - 1);
        const unsigned peers = __match_any_sync(kFull, valid ? d : 0xffffffffu);
        uint32_t *c = count + warp * R + d;
        const uint32_t before = valid ? *c : 0u;
        pos[i] = before + __popc(peers & below);
        __syncwarp();
        if (valid && (peers & below) == 0) *c = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: the warps' counts to offsets in warp order, the digit's total
    uint32_t total[D];
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int d = t * D + k;
        uint32_t acc = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = count[w * R + d];
            count[w * R + d] = acc;
            acc += c;
        }
        total[k] = acc;
    }
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < D; ++k) v += total[k];
    const uint32_t inclusive = block_inclusive_scan(v, warp_sums);
    uint32_t first = inclusive - v;
    if (t == kThreads - 1) tile_count = inclusive;
#pragma unroll
    for (int k = 0; k < D; ++k) {
        const int d = t * D + k;
        start[d] = first;
        run[d] = base[d] + offs[(i64)d * nblocks + blockIdx.x];
        first += total[k];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (valid_mask & (1u << i)) {
            const uint32_t d = (key[i] >> shift) & (R - 1);
            pos[i] += start[d] + count[warp * R + d];
        }
    }
    __syncthreads();  // the counts are read: the space takes the sorted tile
    uint32_t *skey = space, *sval = space + kTile;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (valid_mask & (1u << i)) {
            skey[pos[i]] = key[i];
            sval[pos[i]] = val[i];
        }
    }
    __syncthreads();
    const int sorted = (int)tile_count;
    for (int k = t; k < sorted; k += kThreads) {
        const uint32_t kk = skey[k];
        const uint32_t d = (kk >> shift) & (R - 1);
        const uint32_t at = run[d] + ((uint32_t)k - start[d]);
        keys_out[at] = kk;
        vals_out[at] = sval[k];
    }
}

// a + b, componentwise in order.
__device__ __forceinline__ double4 add4(double4 a, double4 b) {
    return make_double4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}

// Warp segmented reduction of the sorted records.  A segment (one cell) wholly inside a
// warp is written to its cell; pieces of segments crossing warp boundaries are left for
// `seg_reduce_chains`: `first` is a warp's leading piece of a segment begun earlier
// (`tail` set when that segment ends in the warp), `last` its trailing piece of a segment
// that begins in the warp and continues (`owner` set).
__global__ void seg_reduce_warps(const uint32_t *__restrict__ K, const uint32_t *__restrict__ I,
                                 const DepositRec *__restrict__ rec, i64 R_host,
                                 const i64 *__restrict__ R_dev, uint32_t sentinel,
                                 double4 *__restrict__ cells, double4 *__restrict__ first,
                                 double4 *__restrict__ last, uint8_t *__restrict__ tail_flag,
                                 uint8_t *__restrict__ owner_flag, int accumulate) {
    const i64 R = record_count(R_host, R_dev);
    const i64 gw = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (gw * 32 >= R) return;  // whole warps only
    const i64 r = gw * 32 + lane;
    const uint32_t key = r < R ? K[r] : sentinel;
    const bool valid = key < sentinel;
    double c00 = 0.0, c01 = 0.0, c10 = 0.0, c11 = 0.0;
    if (valid) {
        const DepositRec p = rec[I[r]];
        c00 = p.c00;
        c01 = p.c01;
        c10 = p.c10;
        c11 = p.c11;
    }
    const uint32_t prev = (r > 0 && r - 1 < R) ? K[r - 1] : 0xffffffffu;
    const uint32_t next = (r + 1 < R) ? K[r + 1] : 0xffffffffu;
    const bool head = valid && (r == 0 || prev != key);
    const bool tail = valid && (r + 1 >= R || next != key);
    bool f = head;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double y0 = __shfl_up_sync(kFull, c00, off);
        const double y1 = __shfl_up_sync(kFull, c01, off);
        const double y2 = __shfl_up_sync(kFull, c10, off);
        const double y3 = __shfl_up_sync(kFull, c11, off);
        const bool g = __shfl_up_sync(kFull, f, off);
        if (lane >= off) {
            if (!f) {
                c00 = y0 + c00;
                c01 = y1 + c01;
                c10 = y2 + c10;
                c11 = y3 + c11;
            }
            f = f || g;
        }
    }
    const double4 sum = make_double4(c00, c01, c10, c11);
    if (tail) {
        if (f) {
            cells[key] = accumulate ? add4(cells[key], sum) : sum;
        } else {
            first[gw] = sum;
            tail_flag[gw] = 1;
        }
    }
    if (lane == 31) {
        const bool open = valid && !tail;
        owner_flag[gw] = (open && f) ? 1 : 0;
        if (open && f) last[gw] = sum;
        if (open && !f) {
            first[gw] = sum;
            tail_flag[gw] = 0;
        }
    }
}

// The segments that cross warps: the owning warp's trailing piece plus the following
// warps' leading pieces, added in warp order until the segment ends.
__global__ void seg_reduce_chains(const uint32_t *__restrict__ K, i64 R_host,
                                  const i64 *__restrict__ R_dev, double4 *__restrict__ cells,
                                  const double4 *__restrict__ first,
                                  const double4 *__restrict__ last,
                                  const uint8_t *__restrict__ tail_flag,
                                  const uint8_t *__restrict__ owner_flag, int accumulate) {
    const i64 n_warps = (record_count(R_host, R_dev) + 31) / 32;
    const i64 gw = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (gw >= n_warps || !owner_flag[gw]) return;
    double4 s = last[gw];
    for (i64 w = gw + 1; w < n_warps; ++w) {
        const double4 p = first[w];
        s.x = s.x + p.x;
        s.y = s.y + p.y;
        s.z = s.z + p.z;
        s.w = s.w + p.w;
        if (tail_flag[w]) break;
    }
    const uint32_t key = K[gw * 32 + 31];
    cells[key] = accumulate ? add4(cells[key], s) : s;
}

// charge[node] += the four cells around it, in the fixed order (i, j), (i, j-1), (i-1, j),
// (i-1, j-1): the corners (0,0), (0,1), (1,0), (1,1) of those cells.
__global__ void node_accumulate(const double4 *__restrict__ cells, double *__restrict__ charge,
                                const i64 *__restrict__ patch_int, i64 n_patches, i64 nx0,
                                i64 ny0, i64 n_nodes, int ascending) {
    const i64 node = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= n_nodes) return;
    i64 ny = ny0, offset = 0;
    if (patch_int && ascending) {
        // the last patch whose first node is at or before this one
        i64 lo = 0, hi = n_patches - 1;
        while (lo < hi) {
            const i64 mid = (lo + hi + 1) / 2;
            if (__ldg(patch_int + mid * 6 + 5) <= node)
                lo = mid;
            else
                hi = mid - 1;
        }
        ny = __ldg(patch_int + lo * 6 + 1);
        offset = __ldg(patch_int + lo * 6 + 5);
    } else if (patch_int) {
        for (i64 p = 0; p < n_patches; ++p) {
            const i64 off = patch_int[p * 6 + 5];
            if (node >= off && node < off + patch_int[p * 6 + 4]) {
                ny = patch_int[p * 6 + 1];
                offset = off;
                break;
            }
        }
    }
    (void)nx0;
    const i64 local = node - offset;
    const i64 i = local / ny, j = local - i * ny;
    double s = cells[node].x;
    if (j >= 1) s = s + cells[node - 1].y;
    if (i >= 1) s = s + cells[node - ny].z;
    if (i >= 1 && j >= 1) s = s + cells[node - ny - 1].w;
    charge[node] += s;
}

// Records of point charges (deposit_trajectories_2d_pyccel.py:28-59).
__global__ void point_records(const double *__restrict__ px, const double *__restrict__ py,
                              const double *__restrict__ q, i64 n, double origin_x,
                              double origin_y, double h, i64 cylindrical, i64 nx, i64 ny,
                              uint32_t *__restrict__ keys, DepositRec *__restrict__ rec) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double x = px[k], y = py[k];
    i64 i = (i64)floor((x - origin_x) / h);
    i64 j = (i64)floor((y - origin_y) / h);
    double t = (x - (origin_x + h * (double)i)) / h;
    double u;
    if (cylindrical != 0) {
        const double r1 = origin_y + h * (double)j;
        const double r2 = r1 + h;
        u = (y * y - r1 * r1) / (r2 * r2 - r1 * r1);
    } else {
        u = (y - (origin_y + h * (double)j)) / h;
    }
    if (i < 0) {
        t = 0.0;
        i = 0;
    } else if (i >= nx - 1) {
        t = 1.0;
        i = nx - 2;
    }
    if (j < 0) {
        u = 0.0;
        j = 0;
    } else if (j >= ny - 1) {
        u = 1.0;
        j = ny - 2;
    }
    keys[k] = (uint32_t)(i * ny + j);
    const double c = q[k];
    rec[k] = DepositRec{(1.0 - t) * (1.0 - u) * c, (1.0 - t) * u * c, t * (1.0 - u) * c,
                        t * u * c};
}

int bits_for(uint64_t max_key) {
    int b = 0;
    while (b < 32 && (max_key >> b) != 0) ++b;
    return b;
}

}  // namespace

// One stable pass on the digit of R values at `shift`.
// `skip`: the key the pass leaves out; `count`, when not NULL, gets the records it sorted.
template <int R>
void sort_pass(bt_ctx *ctx, const uint32_t *src_k, const uint32_t *src_v, i64 n,
               const i64 *n_dev, uint32_t skip, int shift, uint32_t *hist, uint32_t *offs,
               uint32_t *totals, uint32_t *digit, i64 *count, int nblocks, uint32_t *dst_k,
               uint32_t *dst_v) {
    cudaStream_t st = ctx->stream;
    BT_LAUNCH(ctx, radix_hist<R>, nblocks, kThreads, 0, st, src_k, n, n_dev, skip, shift, hist,
              nblocks);
    BT_LAUNCH(ctx, radix_row_scan, R, kThreads, 0, st, hist, offs, totals, nblocks);
    BT_LAUNCH(ctx, radix_digit_base<R>, 1, kThreads, 0, st, totals, digit, count);
    BT_LAUNCH(ctx, radix_scatter<R>, nblocks, kThreads, 0, st, src_k, src_v, n, n_dev, skip,
              shift, offs, digit, nblocks, dst_k, dst_v);
}

void radix_sort_pairs(bt_ctx *ctx, const uint32_t *keys_in, i64 n, const i64 *n_dev,
                      int key_bits, uint32_t skip, uint32_t **keys_out, uint32_t **vals_out,
                      const i64 **count_out) {
    BT_REQUIRE(n < (i64)0xffffffffLL, "radix sort: too many records for 32-bit indices");
    DepositScratch &s = ctx->deposit;
    const int nblocks = (int)((n + kTile - 1) / kTile);
    uint32_t *ka = s.keys_alt.as<uint32_t>(n), *va = s.vals.as<uint32_t>(n);
    uint32_t *kb = s.keys.as<uint32_t>(n), *vb = s.vals_alt.as<uint32_t>(n);
    uint32_t *hist = s.hist.as<uint32_t>((size_t)kRadixMax * nblocks);
    uint32_t *offs = s.row_offsets.as<uint32_t>((size_t)kRadixMax * nblocks);
    uint32_t *digit = s.digit_base.as<uint32_t>(2 * kRadixMax);
    uint32_t *totals = digit + kRadixMax;
    i64 *sorted = s.sorted.as<i64>(1);  // the records left after the first pass
    const uint32_t *src_k = keys_in;
    const uint32_t *src_v = nullptr;
    uint32_t *dst_k = ka, *dst_v = va;
    BT_REQUIRE(n > 0 && key_bits > 0, "radix sort: nothing to sort");
    // the narrowest of 8-, 9- and 10-bit digits that needs the fewest passes (9 bits for
    // 17-18-bit keys, 10 bits for 19-20; 8 bits otherwise up to 24)
    int bits = 8;
    for (int b = 9; b <= 10; ++b)
        if ((key_bits + b - 1) / b < (key_bits + bits - 1) / bits) bits = b;
    const int passes = (key_bits + bits - 1) / bits;
    // the first pass leaves out the `skip` keys and counts the rest; the later passes sort
    // that many
    for (int p = 0; p < passes; ++p) {
        const int shift = bits * p;
        const i64 *count = p == 0 ? n_dev : sorted;
        const uint32_t leave = p == 0 ? skip : kNoSkip;
        i64 *out = p == 0 ? sorted : nullptr;
        if (bits == 10)
            sort_pass<1024>(ctx, src_k, src_v, n, count, leave, shift, hist, offs, totals,
                            digit, out, nblocks, dst_k, dst_v);
        else if (bits == 9)
            sort_pass<512>(ctx, src_k, src_v, n, count, leave, shift, hist, offs, totals, digit,
                           out, nblocks, dst_k, dst_v);
        else
            sort_pass<256>(ctx, src_k, src_v, n, count, leave, shift, hist, offs, totals, digit,
                           out, nblocks, dst_k, dst_v);
        BT_CHECK_LAUNCH();
        src_k = dst_k;
        src_v = dst_v;
        if (dst_k == ka) {
            dst_k = kb;
            dst_v = vb;
        } else {
            dst_k = ka;
            dst_v = va;
        }
    }
    *keys_out = const_cast<uint32_t *>(src_k);
    *vals_out = const_cast<uint32_t *>(src_v);
    *count_out = sorted;
}

// total += the count of records a sort kept (measurement only: runs while timing is on)
__global__ void add_kept(const i64 *__restrict__ kept, i64 n_records, i64 *__restrict__ total) {
    *total += kept ? *kept : n_records;
}

void deposit_cells_reset(bt_ctx *ctx, i64 n_nodes) {
    double4 *cells = ctx->deposit.cell_sums.as<double4>((size_t)n_nodes);
    BT_CUDA(cudaMemsetAsync(cells, 0, sizeof(double4) * n_nodes, ctx->stream));
}

void deposit_cells_finish(bt_ctx *ctx, double *charge, const NodeLayout &layout) {
    double4 *cells = ctx->deposit.cell_sums.as<double4>((size_t)layout.n_nodes);
    BT_LAUNCH(ctx, node_accumulate, blocks_for(layout.n_nodes, 256), 256, 0, ctx->stream, cells,
              charge, layout.patch_int, layout.n_patches, layout.nx, layout.ny, layout.n_nodes,
              layout.ascending ? 1 : 0);
    BT_CHECK_LAUNCH();
}

void deposit_records(bt_ctx *ctx, const uint32_t *keys, const DepositRec *rec, i64 n_records,
                     const i64 *n_dev, uint32_t sentinel, double *charge,
                     const NodeLayout &layout, bool accumulate) {
    if (n_records == 0) return;
    DepositScratch &s = ctx->deposit;
    cudaStream_t st = ctx->stream;
    uint32_t *sk = nullptr, *sv = nullptr;
    const i64 *n_sorted = nullptr;  // the records with a charge, on the device
    radix_sort_pairs(ctx, keys, n_records, n_dev, bits_for(sentinel), sentinel, &sk, &sv,
                     &n_sorted);
    if (ctx->timing)
        BT_LAUNCH(ctx, add_kept, 1, 1, 0, st, n_sorted, n_records,
                  ctx->kept_records.as<i64>(1));
    const i64 n_warps = (n_records + 31) / 32;
    double4 *cells = s.cell_sums.as<double4>((size_t)layout.n_nodes);
    double4 *first = s.warp_first.as<double4>((size_t)n_warps);
    double4 *last = s.warp_last.as<double4>((size_t)n_warps);
    uint8_t *flags = s.warp_flags.as<uint8_t>((size_t)2 * n_warps);
    if (!accumulate) BT_CUDA(cudaMemsetAsync(cells, 0, sizeof(double4) * layout.n_nodes, st));
    const int threads = 256;
    BT_LAUNCH(ctx, seg_reduce_warps, blocks_for(n_warps * 32, threads), threads, 0, st, sk, sv,
              rec, n_records, n_sorted, sentinel, cells, first, last, flags, flags + n_warps,
              accumulate ? 1 : 0);
    BT_LAUNCH(ctx, seg_reduce_chains, blocks_for(n_warps, threads), threads, 0, st, sk, n_records,
              n_sorted, cells, first, last, flags, flags + n_warps, accumulate ? 1 : 0);
    if (accumulate) {
        BT_CHECK_LAUNCH();
        return;  // the cells carry over to the next deposit; deposit_cells_finish adds them
    }
    BT_LAUNCH(ctx, node_accumulate, blocks_for(layout.n_nodes, threads), threads, 0, st, cells, charge, layout.patch_int, layout.n_patches, layout.nx, layout.ny,
        layout.n_nodes, layout.ascending ? 1 : 0);
    BT_CHECK_LAUNCH();
}

}  // namespace bt

extern "C" int bt_deposit_trajectories_2d(bt_ctx *ctx, const double *px, const double *py,
                                          const double *q, int64_t n, double origin_x,
                                          double origin_y, double h, int64_t cylindrical,
                                          double *charge, int64_t nx, int64_t ny) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx, "deposit: null context");
        BT_REQUIRE(n >= 0, "deposit: negative point count");
        BT_REQUIRE(nx >= 2 && ny >= 2, "deposit: the mesh needs at least 2 x 2 nodes");
        BT_REQUIRE(nx * ny < (int64_t)0xffffffffLL, "deposit: mesh too large for 32-bit keys");
        if (n == 0) return;
        BT_REQUIRE(px && py && q && charge, "deposit: null array");
        bt::DepositScratch &s = ctx->deposit;
        uint32_t *keys = s.keys.as<uint32_t>(n);
        bt::DepositRec *rec = s.rec.as<bt::DepositRec>(n);
        BT_LAUNCH(ctx, bt::point_records, bt::blocks_for(n, 256), 256, 0, ctx->stream, px, py,
                  q, n, origin_x, origin_y, h, cylindrical, nx, ny, keys, rec);
        BT_CHECK_LAUNCH();
        // the records' keys live in `keys`; the sort reads them and writes elsewhere
        bt::NodeLayout layout{nullptr, 1, nx, ny, nx * ny};
        bt::deposit_records(ctx, keys, rec, n, nullptr, (uint32_t)(nx * ny), charge, layout);
    });
}

// -- the deposit without allocation ---------------------------------------------------------
//
// bt_deposit_trajectories_2d_noalloc: the same deterministic deposit for callers that may
// not allocate device memory (their memory is budgeted up front by another allocator, or
// cudaMalloc's implicit device synchronisation is not acceptable where they call).  Its
// scratch is the file-scope array below, of a fixed size; every GPU that loads the library
// holds it until the process exits.  Every call shares it and leaves its last contents
// there: calls that overlap on the GPU (on different streams, or from different host
// threads without ordering) race on it.

namespace bt {
namespace {

constexpr i64 kNoallocPoints = 65536;  // at most this many charges per call
constexpr i64 kNoallocNodes = 65536;   // and a mesh of at most this many nodes
constexpr i64 kNoallocBlocks = (kNoallocPoints + kTile - 1) / kTile;
constexpr i64 kNoallocWarps = (kNoallocPoints + 31) / 32;

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// the carving of the static array, in bytes
constexpr size_t kOffKeys = 0;  // keys, keys_alt, vals, vals_alt (u32)
constexpr size_t kOffPayload = kOffKeys + align256(4 * 4 * kNoallocPoints);  // records
constexpr size_t kOffHist = kOffPayload + align256(32 * kNoallocPoints);  // hist, offs
constexpr size_t kOffDigits = kOffHist + align256(2 * 4 * kRadix * kNoallocBlocks);
constexpr size_t kOffCells = kOffDigits + align256(2 * 4 * kRadix);
constexpr size_t kOffWarps = kOffCells + align256(32 * kNoallocNodes);  // first, last
constexpr size_t kOffFlags = kOffWarps + align256(2 * 32 * kNoallocWarps);
constexpr size_t kNoallocBytes = kOffFlags + align256(2 * kNoallocWarps);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

// The device address of the array in the current device's context, looked up on every
// call: the name itself is only a host-side stand-in, and an address kept from an earlier
// call would dangle once that context is torn down (cudaDeviceReset, or the primary
// context released and made again) and the module loaded anew.  The lookup is a host
// call; the first one in a context may load the module there.
unsigned char *noalloc_scratch() {
    void *address = nullptr;
    BT_CUDA(cudaGetSymbolAddress(&address, g_noalloc_scratch));
    BT_REQUIRE(address != nullptr, "deposit (no allocation): no device address for its scratch");
    return static_cast<unsigned char *>(address);
}

}  // namespace
}  // namespace bt

extern "C" int bt_deposit_trajectories_2d_noalloc(void *stream, const double *px,
                                                  const double *py, const double *q,
                                                  int64_t n, double origin_x, double origin_y,
                                                  double h, int64_t cylindrical, double *charge,
                                                  int64_t nx, int64_t ny) {
    using namespace bt;
    return guarded([&] {
        BT_REQUIRE(n >= 0, "deposit (no allocation): negative point count");
        BT_REQUIRE(nx >= 2 && ny >= 2, "deposit (no allocation): the mesh needs 2 x 2 nodes");
        BT_REQUIRE(n <= kNoallocPoints,
                   "deposit (no allocation): more than 65536 charges in one call exceed its "
                   "static scratch; split the call or use bt_deposit_trajectories_2d");
        BT_REQUIRE(nx * ny <= kNoallocNodes,
                   "deposit (no allocation): a mesh of more than 65536 nodes exceeds its "
                   "static scratch; use bt_deposit_trajectories_2d");
        if (n == 0) return;
        BT_REQUIRE(px && py && q && charge, "deposit (no allocation): null array");
        unsigned char *base = noalloc_scratch();
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        uint32_t *keys = reinterpret_cast<uint32_t *>(base + kOffKeys);
        uint32_t *keys_alt = keys + kNoallocPoints;
        uint32_t *vals = keys_alt + kNoallocPoints;
        uint32_t *vals_alt = vals + kNoallocPoints;
        DepositRec *rec = reinterpret_cast<DepositRec *>(base + kOffPayload);
        uint32_t *hist = reinterpret_cast<uint32_t *>(base + kOffHist);
        uint32_t *offs = hist + kRadix * kNoallocBlocks;
        uint32_t *digit = reinterpret_cast<uint32_t *>(base + kOffDigits);
        uint32_t *totals = digit + kRadix;
        double4 *cells = reinterpret_cast<double4 *>(base + kOffCells);
        double4 *first = reinterpret_cast<double4 *>(base + kOffWarps);
        double4 *last = first + kNoallocWarps;
        uint8_t *flags = base + kOffFlags;
        const uint32_t sentinel = (uint32_t)(nx * ny);

        point_records<<<blocks_for(n, 256), 256, 0, st>>>(px, py, q, n, origin_x, origin_y, h,
                                                          cylindrical, nx, ny, keys, rec);
        // the stable radix sort, ping-ponging between the key and value arrays
        const int nblocks = (int)((n + kTile - 1) / kTile);
        const int passes = (bits_for(sentinel) + 7) / 8;
        const uint32_t *src_k = keys, *src_v = nullptr;
        uint32_t *dst_k = keys_alt, *dst_v = vals;
        for (int pass = 0; pass < passes; ++pass) {
            const int shift = 8 * pass;
            radix_hist<kRadix><<<nblocks, kThreads, 0, st>>>(src_k, n, nullptr, kNoSkip, shift,
                                                             hist, nblocks);
            radix_row_scan<<<kRadix, kThreads, 0, st>>>(hist, offs, totals, nblocks);
            radix_digit_base<kRadix><<<1, kThreads, 0, st>>>(totals, digit, nullptr);
            radix_scatter<kRadix><<<nblocks, kThreads, 0, st>>>(src_k, src_v, n, nullptr, kNoSkip,
                                                                shift,
                                                                offs, digit, nblocks, dst_k,
                                                                dst_v);
            src_k = dst_k;
            src_v = dst_v;
            if (dst_k == keys_alt) {
                dst_k = keys;
                dst_v = vals_alt;
            } else {
                dst_k = keys_alt;
                dst_v = vals;
            }
        }
        // the per-cell sums start at zero; the warp pieces are all written before read
        const i64 n_nodes = nx * ny;
        const i64 n_warps = (n + 31) / 32;
        BT_CUDA(cudaMemsetAsync(cells, 0, sizeof(double4) * n_nodes, st));
        seg_reduce_warps<<<blocks_for(n_warps * 32, 256), 256, 0, st>>>(
            src_k, src_v, rec, n, nullptr, sentinel, cells, first, last, flags,
            flags + n_warps, 0);
        seg_reduce_chains<<<blocks_for(n_warps, 256), 256, 0, st>>>(
            src_k, n, nullptr, cells, first, last, flags, flags + n_warps, 0);
        node_accumulate<<<blocks_for(n_nodes, 256), 256, 0, st>>>(cells, charge, nullptr, 1, nx,
                                                                 ny, n_nodes, 0);
        BT_CHECK_LAUNCH();
    });
}
