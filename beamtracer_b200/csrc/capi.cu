// The context, error reporting and device scratch of the C ABI, and the field gather
// (kernels/staggered_field_2d/staggered_field_2d_pyccel.py:13-55).
#include <map>
#include <mutex>

#include "common.cuh"

namespace bt {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string &message) { g_last_error = message; }

namespace {

constexpr size_t kPoolMaxBytes = (size_t)8 << 30;

constexpr size_t kCarveMax = (size_t)4 << 20;
constexpr size_t kSlabBytes = (size_t)128 << 20;

struct Cached {
    void *ptr;
    bool carved;
};

struct Slab {
    char *base = nullptr;
    size_t used = 0;
};

struct Pool {
    std::mutex mu;
    std::multimap<std::pair<int, size_t>, Cached> blocks;  // (device, bytes) -> block
    size_t cached = 0;                                     // bytes of uncarved blocks
    std::map<int, Slab> slabs;                             // the slab carved from, per device
};

Pool &pool() {
    static Pool p;
    return p;
}

}  // namespace

// A cached block on the current device of at least `need` bytes and at most twice that
// (plus 1 MB), else a new one: a piece of the device's slab for a small block, else its own
// cudaMalloc.
void *pool_take(size_t need, size_t *got, int *device_out, bool *carved) {
    int device = 0;
    cudaGetDevice(&device);
    *device_out = device;
    Pool &p = pool();
    std::lock_guard<std::mutex> lock(p.mu);
    auto it = p.blocks.lower_bound({device, need});
    if (it != p.blocks.end() && it->first.first == device &&
        it->first.second <= 2 * need + ((size_t)1 << 20)) {
        const Cached block = it->second;
        *got = it->first.second;
        if (!block.carved) p.cached -= it->first.second;
        p.blocks.erase(it);
        *carved = block.carved;
        return block.ptr;
    }
    if (need <= kCarveMax) {
        const size_t size = (need + 255) & ~(size_t)255;
        Slab &slab = p.slabs[device];
        if (!slab.base || slab.used + size > kSlabBytes) {
            void *base = nullptr;
            cudaError_t e = cudaMalloc(&base, kSlabBytes);
            if (e != cudaSuccess) {
                (void)cudaGetLastError();
                throw Error{BT_ERR_ALLOC, std::string("cudaMalloc of a slab: ") + cudaGetErrorString(e)};
            }
            slab.base = static_cast<char *>(base);
            slab.used = 0;
        }
        void *ptr = slab.base + slab.used;
        slab.used += size;
        *got = size;
        *carved = true;
        return ptr;
    }
    void *ptr = nullptr;
    cudaError_t e = cudaMalloc(&ptr, need);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw Error{BT_ERR_ALLOC, std::string("cudaMalloc of ") + std::to_string(need) +
                                      " bytes: " + cudaGetErrorString(e)};
    }
    *got = need;
    *carved = false;
    return ptr;
}

void pool_give(void *ptr, size_t bytes, int device, bool carved) {
    if (!ptr) return;
    {
        Pool &p = pool();
        std::lock_guard<std::mutex> lock(p.mu);
        if (carved || p.cached + bytes <= kPoolMaxBytes) {
            p.blocks.insert({{device, bytes}, Cached{ptr, carved}});
            if (!carved) p.cached += bytes;
            return;
        }
    }
    int current = 0;
    cudaGetDevice(&current);
    cudaSetDevice(device);
    cudaFree(ptr);
    cudaSetDevice(current);
}

void *Buffer::get(size_t need) {
    if (need == 0) need = 1;
    if (need <= bytes) return ptr;
    // the old block may still be read by queued work: free it the waiting way (a carved
    // one goes to the cache once the device is idle)
    if (ptr && carved) {
        cudaDeviceSynchronize();
        pool_give(ptr, bytes, device, true);
    } else if (ptr) {
        cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
    size_t got = 0;
    ptr = pool_take(need + need / 4, &got, &device, &carved);
    bytes = got;
    return ptr;
}

void Buffer::release() {
    pool_give(ptr, bytes, device, carved);
    ptr = nullptr;
    bytes = 0;
}

void *HostBuffer::get(size_t need) {
    // at least 64 KB, so that the small read-backs of one call never move the buffer
    if (need < 65536) need = 65536;
    if (need <= bytes) return ptr;
    release();
    cudaError_t e = cudaMallocHost(&ptr, need);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        (void)cudaGetLastError();
        throw Error{BT_ERR_ALLOC, std::string("cudaMallocHost: ") + cudaGetErrorString(e)};
    }
    bytes = need;
    return ptr;
}

void HostBuffer::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

Timed::Timed(bt_ctx *c, const char *name) : ctx(c) {
    if (!ctx || !ctx->timing) return;
    timer = &ctx->timers[name];
    if (!timer->spare.empty()) {
        ev = timer->spare.back();
        timer->spare.pop_back();
    } else {
        cudaEventCreate(&ev.first);
        cudaEventCreate(&ev.second);
    }
    cudaEventRecord(ev.first, ctx->stream);
}

Timed::~Timed() {
    if (!timer) return;
    cudaEventRecord(ev.second, ctx->stream);
    timer->pending.push_back(ev);
}

namespace {

void collect(Timer &t) {
    for (auto &e : t.pending) {
        cudaEventSynchronize(e.second);
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess) {
            t.total_ms += ms;
            t.launches += 1;
        }
        t.spare.push_back(e);
    }
    t.pending.clear();
}

__device__ __forceinline__ double clamped_bilinear(const double *__restrict__ f, i64 nj,
                                                   double s, double t, i64 imax, i64 jmax) {
    i64 i = (i64)floor(s);
    if (i < 0) i = 0;
    if (i > imax) i = imax;
    i64 j = (i64)floor(t);
    if (j < 0) j = 0;
    if (j > jmax) j = jmax;
    const double u = s - (double)i;
    const double w = t - (double)j;
    const double *p = f + i * nj + j;
    const double f00 = __ldg(p), f01 = __ldg(p + 1), f10 = __ldg(p + nj), f11 = __ldg(p + nj + 1);
    const double low = f00 + w * (f01 - f00);
    const double high = f10 + w * (f11 - f10);
    return low + u * (high - low);
}

__global__ void staggered_field(const double *__restrict__ px, const double *__restrict__ py,
                                i64 n, const double *__restrict__ fx,
                                const double *__restrict__ fy, i64 nx, i64 ny, double origin_x,
                                double origin_y, double h, double *__restrict__ ex,
                                double *__restrict__ ey) {
    const i64 k = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double sx = (px[k] - origin_x) / h;
    const double sy = (py[k] - origin_y) / h;
    ex[k] = clamped_bilinear(fx, ny, sx + 0.5, sy, nx - 1, ny - 2);
    ey[k] = clamped_bilinear(fy, ny + 1, sx, sy + 0.5, nx - 2, ny - 1);
}

}  // namespace

}  // namespace bt

extern "C" {

size_t bt_last_error(char *buf, size_t len) {
    const std::string &m = bt::g_last_error;
    if (buf && len) {
        size_t c = m.size() < len - 1 ? m.size() : len - 1;
        memcpy(buf, m.data(), c);
        buf[c] = '\0';
    }
    return m.size();
}

const char *bt_version(void) { return "beamtracer-b200 0.1.0 (sm_100a)"; }

int bt_ctx_create(int device, bt_ctx **out) {
    return bt::guarded([&] {
        BT_REQUIRE(out, "ctx: null out");
        *out = nullptr;
        int count = 0;
        BT_CUDA(cudaGetDeviceCount(&count));
        BT_REQUIRE(device >= 0 && device < count, "ctx: no such CUDA device");
        BT_CUDA(cudaSetDevice(device));
        bt_ctx *ctx = new bt_ctx;
        ctx->device = device;
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete ctx;
            throw bt::Error{BT_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e)};
        }
        ctx->stream = ctx->own_stream;
        cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
        *out = ctx;
    });
}

int bt_ctx_set_timing(bt_ctx *ctx, int on) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx, "ctx: null context");
        if (on && !ctx->timing)  // the record count starts from zero with the timing
            BT_CUDA(cudaMemsetAsync(ctx->kept_records.as<int64_t>(1), 0, sizeof(int64_t),
                                    ctx->stream));
        ctx->timing = on != 0;
    });
}

int bt_ctx_read_timer(bt_ctx *ctx, const char *name, double *total_ms, int64_t *launches) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && name, "ctx: null argument");
        auto it = ctx->timers.find(name);
        double ms = 0.0;
        int64_t count = 0;
        if (it != ctx->timers.end()) {
            bt::collect(it->second);
            ms = it->second.total_ms;
            count = it->second.launches;
        }
        if (total_ms) *total_ms = ms;
        if (launches) *launches = count;
    });
}

int bt_ctx_launch_count(bt_ctx *ctx, int64_t *count) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && count, "ctx: null argument");
        *count = ctx->launch_count;
    });
}

int bt_ctx_reset_timers(bt_ctx *ctx) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx, "ctx: null context");
        for (auto &kv : ctx->timers) {
            bt::collect(kv.second);
            kv.second.total_ms = 0.0;
            kv.second.launches = 0;
        }
        BT_CUDA(cudaMemsetAsync(ctx->kept_records.as<int64_t>(1), 0, sizeof(int64_t),
                                ctx->stream));
    });
}

int bt_ctx_deposit_records(bt_ctx *ctx, int64_t *records) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx && records, "ctx: null argument");
        BT_CUDA(cudaStreamSynchronize(ctx->stream));
        BT_CUDA(cudaMemcpy(records, ctx->kept_records.as<int64_t>(1), sizeof(int64_t),
                           cudaMemcpyDeviceToHost));
    });
}

int bt_ctx_destroy(bt_ctx *ctx) {
    return bt::guarded([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        for (auto &kv : ctx->timers) {
            bt::collect(kv.second);
            for (auto &e : kv.second.spare) {
                cudaEventDestroy(e.first);
                cudaEventDestroy(e.second);
            }
        }
        bt::TraceScratch &ts = ctx->trace;
        if (ts.side) cudaStreamSynchronize(ts.side);
        for (int b = 0; b < 2; ++b) {
            if (ts.filled[b]) cudaEventDestroy(ts.filled[b]);
            if (ts.drained[b]) cudaEventDestroy(ts.drained[b]);
        }
        if (ts.side) cudaStreamDestroy(ts.side);
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
        delete ctx;
    });
}

int bt_ctx_set_stream(bt_ctx *ctx, void *stream) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx, "ctx: null context");
        ctx->stream = static_cast<cudaStream_t>(stream);  // NULL: CUDA's default stream
    });
}

int bt_ctx_synchronize(bt_ctx *ctx) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx, "ctx: null context");
        BT_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int bt_staggered_field_2d(bt_ctx *ctx, const double *px, const double *py, int64_t n,
                          const double *fx, const double *fy, int64_t nx, int64_t ny,
                          double origin_x, double origin_y, double h, double *ex, double *ey) {
    return bt::guarded([&] {
        BT_REQUIRE(ctx, "gather: null context");
        BT_REQUIRE(n >= 0, "gather: negative point count");
        BT_REQUIRE(nx >= 2 && ny >= 2, "gather: the mesh needs at least 2 x 2 nodes");
        if (n == 0) return;
        BT_REQUIRE(px && py && fx && fy && ex && ey, "gather: null array");
        bt::Timed timed(ctx, "staggered_field_2d");
        BT_LAUNCH(ctx, bt::staggered_field, bt::blocks_for(n, 256), 256, 0, ctx->stream, px, py, n, fx, fy, nx, ny, origin_x, origin_y, h, ex, ey);
        BT_CHECK_LAUNCH();
    });
}

}  // extern "C"
