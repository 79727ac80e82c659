// Shared declarations of the beamtracer-b200 CUDA library: the context, device scratch,
// error reporting and the small device helpers every kernel file uses.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/bt200.h"

typedef int64_t i64;

namespace bt {

// -- errors --------------------------------------------------------------------------------

void set_error(const std::string &message);

struct Error {
    int code;
    std::string message;
};

#define BT_CUDA(call)                                                                     \
    do {                                                                                  \
        cudaError_t bt_e_ = (call);                                                       \
        if (bt_e_ != cudaSuccess)                                                         \
            throw ::bt::Error{BT_ERR_CUDA, std::string(#call) + " (" + __FILE__ + ":" +   \
                                               std::to_string(__LINE__) + "): " +         \
                                               cudaGetErrorString(bt_e_)};                \
    } while (0)

#define BT_CHECK_LAUNCH() BT_CUDA(cudaGetLastError())

// Launch a kernel on the context's behalf and count it (one statement).
#define BT_LAUNCH(ctx, kernel, grid, block, smem, stream, ...)                              \
    do {                                                                                  \
        ++(ctx)->launch_count;                                                            \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                       \
    } while (0)

#define BT_REQUIRE(cond, msg)                                                             \
    do {                                                                                  \
        if (!(cond)) throw ::bt::Error{BT_ERR_ARG, (msg)};                                \
    } while (0)

// -- device scratch ------------------------------------------------------------------------

// A growable device buffer owned by a context (grown with cudaMalloc, never shrunk).
// Move-only: a copy would free the same memory twice.
// Device memory of a context or solver.  Growing a buffer frees its old block at once
// (cudaFree waits for the work that may still use it); a destroyed buffer's block goes to a
// per-device cache that later buffers draw from, since its owners (a solver, a context)
// synchronise their stream before they destroy their buffers.  The cache keeps at most
// kPoolMaxBytes; cudaMalloc and cudaFree stay off the path of a solver made and dropped
// per call.
// Blocks of at most 4 MB are carved from 128 MB slabs (one cudaMalloc for many of a
// solver's arrays); a carved block is never freed, only cached.
void *pool_take(size_t need, size_t *got, int *device, bool *carved);
void pool_give(void *ptr, size_t bytes, int device, bool carved);

struct Buffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    int device = 0;       // where the block lives
    bool carved = false;  // a slab's piece (pool_take)
    Buffer() = default;
    Buffer(const Buffer &) = delete;
    Buffer &operator=(const Buffer &) = delete;
    Buffer(Buffer &&o) noexcept : ptr(o.ptr), bytes(o.bytes), device(o.device), carved(o.carved) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    Buffer &operator=(Buffer &&o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            bytes = o.bytes;
            device = o.device;
            carved = o.carved;
            o.ptr = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    void *get(size_t need);
    template <class T>
    T *as(size_t count) {
        return static_cast<T *>(get(count * sizeof(T)));
    }
    void release();
    ~Buffer() { release(); }
};

// Pinned host memory for small read-backs.
struct HostBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    HostBuffer() = default;
    HostBuffer(const HostBuffer &) = delete;
    HostBuffer &operator=(const HostBuffer &) = delete;
    void *get(size_t need);
    void release();
    ~HostBuffer() { release(); }
};

// The scratch of the deterministic deposit (records, their radix sort, per-cell sums).
struct DepositScratch {
    Buffer keys, keys_alt, vals, vals_alt, rec;
    Buffer hist, row_offsets, digit_base, sorted;
    Buffer cell_sums, warp_first, warp_last, warp_flags;
};

// The tracer's scratch: the live lists and two record buffers, one filled by the trace
// windows while the other's records are deposited on the side stream.
struct TraceScratch {
    Buffer active_a, active_b, block_counts, n_alive, alive;
    Buffer rec_keys[2], rec[2];
    cudaStream_t side = nullptr;                 // the deposits' stream
    cudaEvent_t filled[2] = {nullptr, nullptr};  // a buffer's windows are traced
    cudaEvent_t drained[2] = {nullptr, nullptr}; // a buffer's records are deposited
};

}  // namespace bt

namespace bt {
// The launch times of one named kernel (or group of launches): CUDA events recorded on
// the context's stream around each launch, read back and summed on request.
struct Timer {
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending, spare;
    double total_ms = 0.0;
    i64 launches = 0;
};
}  // namespace bt

struct bt_ctx {
    int device = 0;
    bool timing = false;
    std::map<std::string, bt::Timer> timers;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int num_sms = 148;
    bt::DepositScratch deposit;
    bt::TraceScratch trace;
    bt::HostBuffer host;
    bt::Buffer reduce_partial;  // per-block partial results of the device reductions
    bt::Buffer kept_records;    // (device i64) records the deposits reduced while timing
    bt::Buffer anderson;        // the Anderson mixer's sums, R, Q^T f and gamma
    bt::Buffer measure;         // the FP64 peak measurement's output
    // the 3D tracer's records (charge, current), live flags and live count
    bt::Buffer t3_keys, t3_vals, t3_jkeys, t3_jvals, t3_alive, t3_live, t3_cells;
    i64 launch_count = 0;       // kernels launched on the context since its creation
    i64 last_windows = 0, last_records = 0, last_flushes = 0;
};

namespace bt {

// Records the launches between its construction and destruction under `name` when the
// context's timing is on.
struct Timed {
    bt_ctx *ctx;
    Timer *timer = nullptr;
    std::pair<cudaEvent_t, cudaEvent_t> ev{};
    Timed(bt_ctx *c, const char *name);
    ~Timed();
};

// Run `body` and map exceptions to an error code and message.
template <class F>
int guarded(F &&body) {
    try {
        body();
        return BT_OK;
    } catch (const Error &e) {
        set_error(e.message);
        return e.code;
    } catch (const std::exception &e) {
        set_error(e.what());
        return BT_ERR_ALLOC;
    }
}

inline unsigned blocks_for(i64 n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

// -- device helpers --------------------------------------------------------------------------

// The radius sqrt(y^2 + z^2), formed by that expression (the oracle forms it the same way).
__device__ __forceinline__ double radius(double y, double z) { return sqrt(y * y + z * z); }

// The reciprocal that `div_known` divides by b with: 1 / b rounded to nearest, or 0 (plain
// division) for a b outside [2^-60, 2^60] or not a number.
__host__ __device__ __forceinline__ double known_reciprocal(double b) {
    return (b >= 0x1p-60 && b <= 0x1p60) ? 1.0 / b : 0.0;
}

// a / b rounded to nearest, as the IEEE division, for a divisor whose reciprocal
// rb = known_reciprocal(b) is known in advance: the quotient a rb and two corrections by the
// exact remainder.  Markstein's theorem (P. W. Markstein, IBM J. Res. Develop. 34(1), 1990):
// if rb is within half an ulp of 1/b and q within one ulp of a/b, the remainder a - b q is
// exact and q + (a - b q) rb rounds to a/b rounded to nearest.  a rb is within 1.5 ulp of
// a/b, its correction within one, the second correction the rounded quotient.  The
// remainders stay normal and the quotients finite for 2^-900 <= |a| <= 2^900 and
// 2^-60 <= b <= 2^60; any other a (zero, subnormal, huge, infinite, NaN) or b takes the
// IEEE division, so the result is a / b for every a and b.
__device__ __forceinline__ double div_known(double a, double b, double rb) {
    const double m = fabs(a);
    if (rb == 0.0 || !(m >= 0x1p-900 && m <= 0x1p900)) return a / b;
    double q = a * rb;
    double r = fma(-q, b, a);
    q = fma(r, rb, q);
    r = fma(-q, b, a);
    return fma(r, rb, q);
}

// The Lorentz factor sqrt(1 + |u|^2 / c^2) of a proper velocity u (1 for inv_c2 = 0).
__device__ __forceinline__ double lorentz(double u0, double u1, double u2, double inv_c2) {
    return sqrt(1.0 + (u0 * u0 + u1 * u1 + u2 * u2) * inv_c2);
}

// -- electrode shapes (geometry.cu's classification, the batched trace's electrode test) ------

// shape kinds; 3 is an aperture (a polygon and its mirror image)
constexpr int kShapeRect = 0, kShapeCircle = 1, kShapePolygon = 2;
constexpr int kEdgeWords = 9;  // x1, y1, x2, y2, threshold, x_lo, x_hi, y_lo, y_hi

// The tests round every operation as written (explicit _rn operations: the same bits in a
// build that contracts multiply-adds), as the host's NumPy tests do.

// Inside the polygon at p (p[0] its edge count, then its edges) or on its boundary.
__device__ inline bool polygon_inside(const double *__restrict__ p, double x, double y) {
    const i64 n = (i64)p[0];
    const double *e = p + 1;
    bool inside = false, boundary = false;
    for (i64 k = 0; k < n; ++k, e += kEdgeWords) {
        const double x1 = e[0], y1 = e[1], x2 = e[2], y2 = e[3];
        if ((y1 > y) != (y2 > y)) {
            const double at = __dadd_rn(x1, __ddiv_rn(__dmul_rn(y - y1, x2 - x1), y2 - y1));
            if (x < at) inside = !inside;
        }
        const double cross = __dsub_rn(__dmul_rn(x2 - x1, y - y1), __dmul_rn(y2 - y1, x - x1));
        if (fabs(cross) <= e[4] && x >= e[5] && x <= e[6] && y >= e[7] && y <= e[8])
            boundary = true;
    }
    return inside || boundary;
}

__device__ inline bool shape_inside(int kind, const double *__restrict__ p, double x, double y) {
    if (kind == kShapeRect) return fabs(x - p[0]) <= p[2] && fabs(y - p[1]) <= p[3];
    if (kind == kShapeCircle) {
        const double dx = x - p[0], dy = y - p[1];
        return __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= p[2];
    }
    if (kind == kShapePolygon) return polygon_inside(p, x, y);
    // an aperture: the polygon and its mirror image, one after the other
    const bool first = polygon_inside(p, x, y);
    const double *q = p + 1 + (i64)p[0] * kEdgeWords;
    return first || polygon_inside(q, x, y);
}

struct Shapes {
    i64 count;
    const int32_t *kind;
    const i64 *offset;
    const double *params;
};

// The first electrode holding (x, y), or -1 (mesh.inside_solid).
__device__ inline i64 inside_solid(const Shapes &S, double x, double y) {
    for (i64 s = 0; s < S.count; ++s)
        if (shape_inside(S.kind[s], S.params + S.offset[s], x, y)) return s;
    return -1;
}

// -- the deterministic deposit (deposit.cu) ---------------------------------------------------

// Records: key[r] = the lower-left node of the cell the contribution goes to (or
// `sentinel` for none), with its area weights (u along x, w along y) and charge q.
// Sort by key (stable) and add every cell's contributions in record order into its
// four nodes of `charge`; `node_patch` describes how keys map to nodes.
struct NodeLayout {
    const i64 *patch_int;  // (n_patches, 6) as the trace kernel's, device; NULL: one patch
    i64 n_patches;
    i64 nx, ny;            // the single patch's shape when patch_int is NULL
    i64 n_nodes;
    bool ascending = false;  // the patches' node ranges follow one another (a batch of
                             // candidates): a node's patch is found by bisection
};

// A record's payload: the charge it adds to the four nodes of its cell, (i, j), (i, j+1),
// (i+1, j) and (i+1, j+1), in one 32-byte sector so that the reduction's gather through the
// sort permutation reads one sector per record.
struct __align__(32) DepositRec {
    double c00, c01, c10, c11;
};

// n_records sizes the launches; n_dev, when not NULL, is the device-held count of the
// records to deposit (at most n_records): the first ones, the rest ignored.
// accumulate: the per-cell sums are added to those of the deposits before (no node charges
// yet): deposit_cells_reset zeroes them, deposit_cells_finish adds them to the nodes once.
void deposit_records(bt_ctx *ctx, const uint32_t *keys, const DepositRec *rec, i64 n_records,
                     const i64 *n_dev, uint32_t sentinel, double *charge,
                     const NodeLayout &layout, bool accumulate = false);
void deposit_cells_reset(bt_ctx *ctx, i64 n_nodes);
void deposit_cells_finish(bt_ctx *ctx, double *charge, const NodeLayout &layout);

// Stable LSD radix sort of (key, index) pairs: sorted keys and the permutation, leaving
// out the keys equal to `skip`.  Returns the device pointers of the sorted keys and values
// (inside the scratch) and of the device-held count of sorted pairs.  n sizes the
// launches; n_dev, when not NULL, is the device-held count of keys to sort (at most n).
void radix_sort_pairs(bt_ctx *ctx, const uint32_t *keys_in, i64 n, const i64 *n_dev,
                      int key_bits, uint32_t skip, uint32_t **keys_out, uint32_t **vals_out,
                      const i64 **count_out);

}  // namespace bt
