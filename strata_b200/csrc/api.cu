// api.cu - the C ABI of libstrata_cuda (include/strata_cuda.h).
//
// The host side of the device backend: the checks exec.ProcessN makes
// before it runs (internal/exec/process.go:37-135), staging of host
// rasters through device memory, the launches, Stats, and the stage
// builders that resolve the typed options as the terrain, focal and
// transfer packages do.
#include <cuda_runtime.h>

#include <unistd.h>

#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <functional>
#include <thread>
#include <future>
#include <thread>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "launch.h"

using strata::EpiStage;
using strata::LaunchParams;
using strata::ValidityParams;

// ---------------------------------------------------------------------------
// Errors.

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? STRATA_ENOMEM : STRATA_ECUDA, "strata_cuda: %s: %s", what,
                cudaGetErrorString(e));
}

// Go's %v for a float64 (fmt: the shortest representation that round
// trips, %e form when the exponent is < -4 or >= 21), or for a float32
// with f32 set. Used to reproduce the reference's panic messages.
std::string fmt_v(double x, bool f32 = false) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x > 0 ? "+Inf" : "-Inf";
    if (x == 0) return std::signbit(x) ? "-0" : "0";
    char buf[64];
    int prec = 1;
    for (; prec <= 17; prec++) {
        snprintf(buf, sizeof buf, "%.*e", prec - 1, x);
        double back = strtod(buf, nullptr);
        if (f32 ? (float)back == (float)x : back == x) break;
    }
    snprintf(buf, sizeof buf, "%.*e", prec - 1, x);
    // buf: d.ddde[+-]XX
    std::string s(buf);
    size_t e = s.find('e');
    int exp = atoi(s.c_str() + e + 1);
    std::string digits;
    for (size_t i = 0; i < e; i++)
        if (isdigit((unsigned char)s[i])) digits += s[i];
    bool neg = x < 0;
    std::string out = neg ? "-" : "";
    if (exp < -4 || exp >= 21) {
        out += digits.substr(0, 1);
        if (digits.size() > 1) out += "." + digits.substr(1);
        char eb[16];
        snprintf(eb, sizeof eb, "e%c%02d", exp < 0 ? '-' : '+', exp < 0 ? -exp : exp);
        out += eb;
        return out;
    }
    if (exp < 0) {
        out += "0." + std::string(-exp - 1, '0') + digits;
    } else if ((int)digits.size() <= exp + 1) {
        out += digits + std::string(exp + 1 - digits.size(), '0');
    } else {
        out += digits.substr(0, exp + 1) + "." + digits.substr(exp + 1);
    }
    return out;
}

}  // namespace

// ---------------------------------------------------------------------------
// The caller's current device, put back when an entry point returns. Each
// entry point makes its context's device current for its CUDA calls; the
// guard restores the caller's device afterwards, unless the caller's
// thread had no context on it (then restoring would create one, with its
// memory, on a device the caller never used).

namespace {

using PrimaryCtxStateFn = int (*)(int, unsigned int*, int*);  // cuDevicePrimaryCtxGetState

bool primary_active(int dev) {
    static PrimaryCtxStateFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuDevicePrimaryCtxGetState", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PrimaryCtxStateFn>(p);
    }();
    unsigned int flags = 0;
    int active = 0;
    return fn && fn(dev, &flags, &active) == 0 && active;
}

struct DeviceGuard {
    int prev = -1, dev;
    explicit DeviceGuard(int d) : dev(d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceGuard() {
        if (prev >= 0 && prev != dev && primary_active(prev)) cudaSetDevice(prev);
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// Context.

struct strata_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // device-to-host copies that overlap the next kernel
    std::mutex mu;
    // Device buffers for host operands, grown on demand and reused.
    struct Buf {
        void* p = nullptr;
        size_t n = 0;
    };
    std::vector<Buf> bufs;
    // Page-locked staging of the first and last mask words of host
    // destinations (two a destination), merged into the caller's words.
    uint64_t* h_edges = nullptr;
    size_t n_edges = 0;
    // A device word kernels set when a bounded wait runs out, and its
    // page-locked host copy.
    int* d_status = nullptr;
    int* h_status = nullptr;
    // The chunked calls' two tile buffer sets (page-locked and device),
    // grown on demand and reused.
    std::shared_ptr<void> chunk_sets;
    // A second compute stream for the features of one Features call that
    // run as their own launches (one kernel's tail overlaps the next's
    // start), with the events that fork it from and join it back to the
    // call's stream; made on first use.
    cudaStream_t aux_stream = nullptr;
    cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
};

namespace {

// Context buffer slots: 0 and 1 a host source's cells and mask, 2 + 2i
// and 3 + 2i host destination i's, kInputSlot + 2j and the next a further
// host source j's; from kFitScratchSlot the raw sums of Wood's fit.
constexpr int kFitScratchSlot = 128;
// From kInputSlot + 2j: a host source j >= 1's cells and mask.
constexpr int kInputSlot = 8;

int ensure(strata_ctx* c, int slot, size_t bytes, void** out) {
    if ((int)c->bufs.size() <= slot) c->bufs.resize(slot + 1);
    auto& b = c->bufs[slot];
    if (b.n < bytes) {
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.n = 0;
        size_t want = bytes + bytes / 8 + 256;
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return cuda_fail(e, "device buffer");
        }
        b.n = want;
    }
    *out = b.p;
    return STRATA_OK;
}

}  // namespace

extern "C" int strata_abi_version(void) { return STRATA_ABI_VERSION; }

extern "C" const char* strata_last_error(void) { return g_err.c_str(); }

extern "C" int strata_ctx_create(int device, strata_ctx** out) {
    if (!out) return fail(STRATA_EINVAL, "strata_cuda: nil output pointer");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= n) return fail(STRATA_EINVAL, "strata_cuda: device %d out of range [0, %d)", device, n);
    DeviceGuard device_guard(device);
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    auto* c = new strata_ctx;
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->d_status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaHostAlloc(&c->h_status, sizeof(int), cudaHostAllocDefault);
    if (e != cudaSuccess) {
        strata_ctx_destroy(c);
        return cuda_fail(e, "context set-up");
    }
    *c->h_status = 0;
    *out = c;
    return STRATA_OK;
}

extern "C" void strata_ctx_destroy(strata_ctx* c) {
    if (!c) return;
    DeviceGuard device_guard(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto& b : c->bufs)
        if (b.p) cudaFree(b.p);
    if (c->d_status) cudaFree(c->d_status);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->h_edges) cudaFreeHost(c->h_edges);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    if (c->aux_fork) cudaEventDestroy(c->aux_fork);
    if (c->aux_join) cudaEventDestroy(c->aux_join);
    delete c;
}

extern "C" int strata_ctx_device(const strata_ctx* c) { return c ? c->device : -1; }

namespace {

// Reads and clears the status word after the work on st: STRATA_OK, or
// the code a kernel recorded (STRATA_ETIMEDOUT).
int take_status(strata_ctx* c, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(c->h_status, c->d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "kernel");
    int code = *c->h_status;
    if (code != 0) {
        cudaMemsetAsync(c->d_status, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return fail(code, "strata_cuda: a device-side wait ran out (status %d)", code);
    }
    return STRATA_OK;
}

}  // namespace

extern "C" int strata_ctx_synchronize(strata_ctx* c) {
    if (!c) return fail(STRATA_EINVAL, "strata_cuda: nil context");
    DeviceGuard device_guard(c->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
    return take_status(c, c->stream);
}

extern "C" int strata_alloc(strata_ctx* c, size_t bytes, void** dev) {
    if (!c || !dev) return fail(STRATA_EINVAL, "strata_cuda: nil argument");
    DeviceGuard device_guard(c->device);
    cudaError_t e = cudaMalloc(dev, bytes ? bytes : 1);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "cudaMalloc");
    }
    return STRATA_OK;
}

extern "C" int strata_free(strata_ctx* c, void* dev) {
    if (!c) return fail(STRATA_EINVAL, "strata_cuda: nil context");
    DeviceGuard device_guard(c->device);
    cudaError_t e = cudaFree(dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFree");
    return STRATA_OK;
}

extern "C" int strata_upload(strata_ctx* c, void* dev, const void* host, size_t bytes) {
    if (!c) return fail(STRATA_EINVAL, "strata_cuda: nil context");
    DeviceGuard device_guard(c->device);
    cudaError_t e = cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "upload");
    return STRATA_OK;
}

extern "C" int strata_download(strata_ctx* c, void* host, const void* dev, size_t bytes) {
    if (!c) return fail(STRATA_EINVAL, "strata_cuda: nil context");
    DeviceGuard device_guard(c->device);
    cudaError_t e = cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(e, "download");
    return STRATA_OK;
}

// ---------------------------------------------------------------------------
// Checks of ProcessN (internal/exec/process.go:37-135).

namespace {

int64_t span_cells(const strata_raster& r) { return (r.height - 1) * r.stride + r.width; }

// raster.Float32Raster.Validate (raster/raster.go:174-203), for the
// fields a C caller passes.
int validate(const char* name, int i, const strata_raster& r) {
    if (r.width <= 0 || r.height <= 0)
        return fail(STRATA_EINVAL, "engine: %s[%d]: raster: dimensions must be positive, got %lld×%lld", name, i,
                    (long long)r.width, (long long)r.height);
    if (r.stride < r.width)
        return fail(STRATA_EINVAL, "engine: %s[%d]: raster: stride %lld is less than width %lld", name, i,
                    (long long)r.stride, (long long)r.width);
    if (r.height - 1 > (INT64_MAX - r.width) / r.stride)
        return fail(STRATA_EINVAL, "engine: %s[%d]: raster: %lld×%lld with stride %lld has more cells than an int holds",
                    name, i, (long long)r.width, (long long)r.height, (long long)r.stride);
    if (!r.data) return fail(STRATA_EINVAL, "engine: %s[%d]: raster: nil Data", name, i);
    if (r.valid && r.valid_offset < 0)
        return fail(STRATA_EINVAL, "engine: %s[%d]: raster: negative ValidOffset %lld", name, i,
                    (long long)r.valid_offset);
    return STRATA_OK;
}

enum Relation { kDisjoint, kSame, kPartial };

bool spans_meet(int64_t a0, int64_t an, int64_t b0, int64_t bn) { return a0 < b0 + bn && b0 < a0 + an; }

// overlap.relate (internal/overlap/overlap.go).
Relation relate(int64_t a0, int64_t as, int64_t b0, int64_t bs, int64_t w, int64_t h) {
    if (!spans_meet(a0, (h - 1) * as + w, b0, (h - 1) * bs + w)) return kDisjoint;
    if (a0 == b0) return (as == bs || h == 1) ? kSame : kPartial;
    if (as != bs) return kPartial;
    int64_t diff = a0 - b0;
    int64_t dy = diff / as, dx = diff % as;
    if (dx < 0) {
        dy -= 1;
        dx += as;
    }
    auto rows_meet = [h](int64_t d) { return d > -h && d < h; };
    if ((dx < w && rows_meet(dy)) || (dx > as - w && rows_meet(dy + 1))) return kPartial;
    return kDisjoint;
}

// Two operands can only share memory when they are in the same address
// space: both on the device or both on the host.
bool same_space(const strata_raster& a, const strata_raster& b) { return (a.on_device != 0) == (b.on_device != 0); }

Relation data_rel(const strata_raster& a, const strata_raster& b) {
    if (!same_space(a, b)) return kDisjoint;
    int64_t a0 = (int64_t)(uintptr_t)a.data, b0 = (int64_t)(uintptr_t)b.data;
    if ((a0 - b0) % 4 != 0) return spans_meet(a0, span_cells(a) * 4, b0, span_cells(b) * 4) ? kPartial : kDisjoint;
    return relate(a0 / 4, a.stride, b0 / 4, b.stride, a.width, a.height);
}

int64_t bit_addr(const strata_raster& r) { return (int64_t)(uintptr_t)r.valid * 8 + r.valid_offset; }

Relation bits_rel(const strata_raster& a, const strata_raster& b) {
    if (!a.valid || !b.valid || !same_space(a, b)) return kDisjoint;
    return relate(bit_addr(a), a.stride, bit_addr(b), b.stride, a.width, a.height);
}

bool data_spans(const strata_raster& a, const strata_raster& b) {
    if (!same_space(a, b)) return false;
    return spans_meet((int64_t)(uintptr_t)a.data, span_cells(a) * 4, (int64_t)(uintptr_t)b.data, span_cells(b) * 4);
}

bool bit_spans(const strata_raster& a, const strata_raster& b) {
    if (!a.valid || !b.valid || !same_space(a, b)) return false;
    return spans_meet(bit_addr(a), span_cells(a), bit_addr(b), span_cells(b));
}

// vec.Op's names (internal/vec/chain.go:45-51).
const char* vec_name(int op) {
    static const char* const names[] = {"Add",    "Sub",     "Mul",   "Div", "Min", "Max", "AddScalar",
                                        "MulScalar", "Affine", "SubDiv", "Clamp", "Abs", "Sqrt"};
    return op >= 0 && op <= STRATA_VEC_SQRT ? names[op] : "Op";
}

bool is_pointwise(uint32_t op) { return op == STRATA_OP_LOOKUP || op == STRATA_OP_RECLASS || op == STRATA_OP_STEP; }
bool binary_step(int op) { return op >= STRATA_VEC_ADD && op <= STRATA_VEC_MAX; }

// vec.NewChain's step checks (internal/vec/chain.go:106-132).
int check_step(int op, int input) {
    if (op < STRATA_VEC_ADD || op > STRATA_VEC_SQRT)
        return fail(STRATA_EINVAL, "vec: chain step has unknown operation Op(%d)", op);
    if (binary_step(op) && (input < 0 || input >= STRATA_MAX_INPUTS))
        return fail(STRATA_EINVAL, "vec: chain step (%s) reads input %d, which is not one of its %d", vec_name(op),
                    input, STRATA_MAX_INPUTS);
    if (!binary_step(op) && input != -1)
        return fail(STRATA_EINVAL, "vec: chain step (%s) reads no input, so its Src must be -1, not %d", vec_name(op),
                    input);
    return STRATA_OK;
}

int op_radius(const strata_stage& s) {
    if (s.flags & STRATA_STAGE_FIT) return s.radius;
    switch (s.op) {
    case STRATA_OP_HEATLOAD:
    case STRATA_OP_ORIENTATION:
    case STRATA_OP_GRADIENT:
    case STRATA_OP_SLOPE:
    case STRATA_OP_ASPECT:
    case STRATA_OP_HILLSHADE:
    case STRATA_OP_CURVATURE:
        return 1;
    case STRATA_OP_LOOKUP:
    case STRATA_OP_RECLASS:
        return 0;
    default:
        return s.radius;
    }
}

bool finite32(float v) { return v - v == 0; }

// A stage's tables into the launch parameters.
int fill_stage(const strata_stage& s, LaunchParams& p, int epi_index) {
    if (s.op == STRATA_OP_STEP) {
        int rc = check_step(s.kind, s.input);
        if (rc) return rc;
        if (p.nstep >= STRATA_MAX_STEPS)
            return fail(STRATA_EINVAL, "vec: chain has more than %d steps", STRATA_MAX_STEPS);
        p.step[p.nstep++] = strata::ChainStep{s.kind, binary_step(s.kind) ? s.input : 0, s.k[0], s.k[1]};
        return STRATA_OK;
    }
    if (is_pointwise(s.op)) {
        if (epi_index >= strata::kMaxEpilogue)
            return fail(STRATA_ENOTSUP, "engine: a pipeline on the gpu backend takes at most %d pointwise stages",
                        strata::kMaxEpilogue);
        EpiStage& e = p.epi[epi_index];
        e.op = (int)s.op;
        int n = s.table_len[0];
        if (n < (s.op == STRATA_OP_LOOKUP ? 1 : 0) || n > STRATA_MAX_KNOTS || !s.table[0] || !s.table[1])
            return fail(STRATA_EINVAL, "engine: stage table of %d entries (1 to %d)", n, STRATA_MAX_KNOTS);
        e.n = n;
        // transfer.checkIncreasing (transfer/transfer.go:225-239): the
        // device's table index relies on strictly increasing knots.
        for (int i = 0; i < n; i++)
            if (s.table[0][i] != s.table[0][i] || (i > 0 && !(s.table[0][i - 1] < s.table[0][i])))
                return fail(STRATA_EINVAL, "engine: %s table must be strictly increasing and free of NaN",
                            s.op == STRATA_OP_LOOKUP ? "Lookup" : "Reclass");
        memcpy(e.a, s.table[0], sizeof(float) * n);
        memcpy(e.b, s.table[1], sizeof(float) * (s.op == STRATA_OP_LOOKUP ? n : n + 1));
        return STRATA_OK;
    }
    p.op = (int)s.op;
    p.radius = op_radius(s);
    p.kind = s.kind;
    p.fit = 0;
    if (s.flags & STRATA_STAGE_FIT) {
        const bool product = (s.op >= STRATA_OP_GRADIENT && s.op <= STRATA_OP_CURVATURE) ||
                             s.op == STRATA_OP_HEATLOAD || s.op == STRATA_OP_ORIENTATION;
        if (!product || s.radius < 1 || s.radius > STRATA_MAX_RADIUS)
            return fail(STRATA_EINVAL, "terrain: FitRadius must be 0 to %d, got %d", STRATA_MAX_RADIUS, s.radius);
        p.fit = s.radius;
    }
    if (s.op == STRATA_OP_HEATLOAD) {
        if (!s.table[0] || s.table_len[0] != 16)
            return fail(STRATA_EINVAL, "engine: a heat load stage carries its 8 float64 terms in 16 table slots");
        memcpy(p.w, s.table[0], 16 * sizeof(float));
    }
    // Slope and Aspect read their kind as a flag (take the arctangent;
    // trigonometric angles).
    if (s.op == STRATA_OP_SLOPE || s.op == STRATA_OP_ASPECT) p.kind = s.kind != 0;
    memcpy(p.k, s.k, sizeof p.k);
    int r = p.radius;
    if (s.op >= STRATA_OP_RUGGEDNESS && s.op <= STRATA_OP_MAX && (r < 1 || r > STRATA_MAX_RADIUS))
        return fail(STRATA_EINVAL, "engine: stage radius %d outside 1 to %d", r, STRATA_MAX_RADIUS);
    int d = 2 * r + 1;
    if (s.op == STRATA_OP_CORRELATE) {
        if (s.table_len[0] != d * d || !s.table[0])
            return fail(STRATA_EINVAL, "focal: Radius %d needs %d×%d = %d Weights, got %d", r, d, d, d * d,
                        s.table_len[0]);
        for (int i = 0; i < d * d; i++) {
            int j = (s.flags & STRATA_STAGE_ROTATE180) ? d * d - 1 - i : i;
            p.w[j] = s.table[0][i];
        }
    } else if (s.op == STRATA_OP_SEPARABLE) {
        if (s.table_len[0] != d || s.table_len[1] != d || !s.table[0] || !s.table[1])
            return fail(STRATA_EINVAL, "focal: Radius %d needs %d Row and %d Col taps, got %d and %d", r, d, d,
                        s.table_len[0], s.table_len[1]);
        for (int i = 0; i < d; i++) {
            p.w[i] = s.table[0][i];
            p.w[17 + i] = s.table[1][i];
        }
    }
    if (s.op == STRATA_OP_CURVATURE && (s.kind < 0 || s.kind > 2))
        return fail(STRATA_EINVAL, "stencil: unknown CurvatureKind %d", s.kind);
    if (s.op == STRATA_OP_RUGGEDNESS && (s.kind < 0 || s.kind > 3))
        return fail(STRATA_EINVAL, "stencil: unknown RuggednessKind %d", s.kind);
    return STRATA_OK;
}

int check_opts(const strata_exec_opts* o) {
    if (o && (o->tile_width < 0 || o->tile_height < 0 || o->workers < 0))
        return fail(STRATA_EINVAL, "engine: negative Options {TileWidth:%lld TileHeight:%lld Workers:%d}",
                    (long long)o->tile_width, (long long)o->tile_height, o->workers);
    return STRATA_OK;
}

// ---------------------------------------------------------------------------
// Folding a pointwise tail that ends in Reclass into one Reclass table.
//
// A Lookup followed by Reclass stages (or Reclass stages alone) maps each
// cell to a step function of its value: between two lookup knots the
// interpolation y0 + (v - x0) / (x1 - x0) * (y1 - y0), each step rounded,
// is monotone in v, so the first Reclass's class index is monotone there
// and changes at a few float thresholds. Those thresholds, found by
// bisection over the floats in order, with the classes' values carried
// through the remaining Reclass stages, form one Reclass table that gives
// every non-NaN cell the same bits as the stages run one after another
// (and NaN passes through both). The host arithmetic below is the
// device's (internal/curve/scalar.go:39-114): IEEE float32 operations
// rounded to nearest, built without contraction.

float host_lookup(float v, const float* xs, const float* ys, int n) {
    int k = 0;
    while (k < n && xs[k] <= v) k++;
    const int lo = k == 0 ? 0 : k - 1, hi = k == n ? n - 1 : k;
    const float x0 = xs[lo], y0 = ys[lo];
    const float t = (v - x0) / (xs[hi] - x0);
    float r = y0 + t * (ys[hi] - y0);
    if (v == x0) r = y0;
    if (k == n) r = ys[n - 1];
    if (k == 0) r = ys[0];
    return v != v ? v : r;
}

int host_class(float v, const float* breaks, int nb) {
    int k = 0;
    while (k < nb && breaks[k] <= v) k++;
    return k;
}

float host_reclass(float v, const float* breaks, int nb, const float* values) {
    return v != v ? v : values[host_class(v, breaks, nb)];
}

// Floats in order as unsigned keys (-0 just below +0), and back.
uint32_t float_key(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
float key_float(uint32_t k) {
    const uint32_t b = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

bool moderate(const float* v, int n) {
    for (int i = 0; i < n; i++)
        if (!(v[i] >= -1e30f && v[i] <= 1e30f)) return false;
    return true;
}

// The fold of p's pointwise stages into one Reclass, if they fold: true
// and the stage in *out, else false.
bool fold_stages(const LaunchParams& p, EpiStage* out) {
    const int n = p.nepi;
    if (n < 2) return false;
    const EpiStage* e = p.epi;
    const bool lookup = e[0].op == STRATA_OP_LOOKUP;
    const int r1 = lookup ? 1 : 0;  // the first Reclass
    for (int i = r1; i < n; i++)
        if (e[i].op != STRATA_OP_RECLASS) return false;
    if (lookup && (!moderate(e[0].a, e[0].n) || !moderate(e[0].b, e[0].n))) return false;
    if (lookup)
        for (int i = 0; i + 1 < e[0].n; i++)
            if (!std::isfinite(e[0].a[i + 1] - e[0].a[i]) || !std::isfinite(e[0].b[i + 1] - e[0].b[i])) return false;
    // The value of class c of the first Reclass after the later ones.
    auto carry = [&](int c) {
        float v = e[r1].b[c];
        for (int i = r1 + 1; i < n; i++) v = host_reclass(v, e[i].a, e[i].n, e[i].b);
        return v;
    };
    auto cls = [&](float v) {
        const float u = lookup ? host_lookup(v, e[0].a, e[0].b, e[0].n) : v;
        return host_class(u, e[r1].a, e[r1].n);
    };
    float brk[STRATA_MAX_KNOTS] = {}, val[STRATA_MAX_KNOTS + 1] = {};
    int nb = 0;
    bool fits = true;
    auto same = [](float a, float b) { return memcmp(&a, &b, 4) == 0; };
    auto step_to = [&](float at, float v) {
        if (same(v, val[nb])) return;
        if (nb == STRATA_MAX_KNOTS) {
            fits = false;
            return;
        }
        brk[nb++] = at;
        val[nb] = v;
    };
    // The pieces on which the class index is monotone: between the
    // lookup's knots (or, with no Lookup, between the first Reclass's
    // breaks, where it is constant).
    const float* knots = lookup ? e[0].a : e[r1].a;
    const int nk = lookup ? e[0].n : e[r1].n;
    const float ninf = -std::numeric_limits<float>::infinity();
    int c = cls(ninf);
    val[0] = carry(c);
    for (int k = 0; k < nk && fits; k++) {
        uint32_t lo = float_key(knots[k]);
        const uint32_t end = k + 1 < nk ? float_key(knots[k + 1]) : float_key(std::numeric_limits<float>::infinity()) + 1;
        c = cls(knots[k]);
        step_to(knots[k], carry(c));
        // the next change of class inside [lo, end): bisect the monotone index
        while (fits && lo + 1 < end && cls(key_float(end - 1)) != c) {
            uint32_t a = lo, b = end - 1;  // cls(a) == c, cls(b) != c
            while (b - a > 1) {
                const uint32_t m = a + (b - a) / 2;
                (cls(key_float(m)) == c ? a : b) = m;
            }
            c = cls(key_float(b));
            step_to(key_float(b), carry(c));
            lo = b;
        }
    }
    if (!fits) return false;
    memset(out, 0, sizeof *out);
    out->op = STRATA_OP_RECLASS;
    out->n = nb;
    memcpy(out->a, brk, sizeof(float) * nb);
    memcpy(out->b, val, sizeof(float) * (nb + 1));
    return true;
}

// Replaces p's pointwise stages by their fold when they fold, remembering
// the last few folds of the calling thread (a fold bisects the floats, a
// cached one is a table compare).
void fold_tail(LaunchParams& p) {
    if (p.nepi < 2 || p.nstep) return;
    struct Entry {
        int nepi = 0;
        EpiStage in[strata::kMaxEpilogue];
        bool folds = false;
        EpiStage out;
    };
    thread_local Entry cache[4];
    thread_local int next = 0;
    const size_t bytes = sizeof(EpiStage) * (size_t)p.nepi;
    for (const Entry& c : cache)
        if (c.nepi == p.nepi && memcmp(c.in, p.epi, bytes) == 0) {
            if (c.folds) {
                p.epi[0] = c.out;
                p.nepi = 1;
            }
            return;
        }
    Entry& c = cache[next];
    next = (next + 1) % 4;
    c.nepi = p.nepi;
    memcpy(c.in, p.epi, bytes);
    c.folds = fold_stages(p, &c.out);
    if (c.folds) {
        p.epi[0] = c.out;
        p.nepi = 1;
    }
}

// ---------------------------------------------------------------------------
// A Slope followed by a lone Reclass (a classification, or the fold above
// of a Lookup -> Reclass tail) as a Reclass of the squared gradient
// magnitude s = gx*gx + gy*gy, the float32 the reference takes the square
// root of (internal/stencil/horn.go:193-222). The slope of s is
// float32(Atan32(sqrt(s)) * scale) (or sqrt(s) * scale without the
// arctangent): the correctly rounded square root is monotone, Atan32 is
// monotone non-decreasing on the non-negative floats (checked on all 2^31
// of them), and a product by a positive scale rounded to nearest is
// monotone, so the slope never falls as s grows. A class break b is then
// reached exactly from the first s whose slope is at or above b, which a
// bisection over the floats finds with the device's arithmetic; the kernel
// compares s with those thresholds and needs no square root, division or
// arctangent. s is a sum of squares, so never negative; a NaN s (a NaN in
// the window) stays NaN as the Reclass leaves it, and a break the slope of
// +Inf does not reach gets a NaN threshold, which no s passes.

// Atan32 (internal/stencil/horn.go:249-262), rounded step by step as the
// device rounds it.
float host_atan32(float x) {
    const float kTan3Pi8 = 0x1.3504f4p+1f, kTanPi8 = 0x1.a8279ap-2f;
    float num = x, den = 1.0f, y0 = 0.0f;
    if (x > kTanPi8) {
        num = x - 1.0f;
        den = x + 1.0f;
        y0 = 0x1.921fb6p-1f;
    }
    if (x > kTan3Pi8) {
        num = -1.0f;
        den = x;
        y0 = 0x1.921fb6p+0f;
    }
    const float t = num / den;
    const float z = t * t;
    float p = 0x1.49e1a2p-4f * z - 0x1.1c370ap-3f;
    p = p * z + 0x1.9924bep-3f;
    p = p * z - 0x1.555454p-2f;
    const float pzt = (p * z) * t;
    return y0 + (pzt + t);
}

float host_slope_of_square(float s, float scale, bool take_atan) {
    const float m = std::sqrt(s);
    return (take_atan ? host_atan32(m) : m) * scale;
}

void fold_slope_square(LaunchParams& p) {
    if (p.op != STRATA_OP_SLOPE || p.nstep || p.nepi != 1 || p.epi[0].op != STRATA_OP_RECLASS) return;
    EpiStage& e = p.epi[0];
    const float scale = p.k[p.fit ? 5 : 2];  // a fit's product constants follow its five factors
    if (e.n > strata::kChainBreaks || !(scale > 0) || std::isinf(scale)) return;
    const bool take_atan = p.kind != 0;
    const float inf = std::numeric_limits<float>::infinity();
    const uint32_t k0 = float_key(0.0f), kinf = float_key(inf);
    for (int j = 0; j < e.n; j++) {
        const float b = e.a[j];
        float t;
        if (host_slope_of_square(inf, scale, take_atan) < b) {
            t = std::numeric_limits<float>::quiet_NaN();
        } else if (host_slope_of_square(0.0f, scale, take_atan) >= b) {
            t = 0.0f;
        } else {
            uint32_t lo = k0, hi = kinf;  // slope(lo) < b <= slope(hi)
            while (hi - lo > 1) {
                const uint32_t m = lo + (hi - lo) / 2;
                (host_slope_of_square(key_float(m), scale, take_atan) >= b ? hi : lo) = m;
            }
            t = key_float(hi);
        }
        e.a[j] = t;
    }
    p.kind = strata::kSlopeSquareClass;
}

// Resolves stages into launch parameters (op, radius, epilogue).
int plan_stages(const strata_stage* stages, int nstages, LaunchParams& p, int* nout) {
    if (!stages || nstages < 1) return fail(STRATA_EINVAL, "engine: nil kernel");
    memset(&p, 0, sizeof p);
    const strata_stage& s0 = stages[0];
    if (s0.op < STRATA_OP_GRADIENT || s0.op > STRATA_OP_STEP)
        return fail(STRATA_EINVAL, "engine: unknown op %u", s0.op);
    int epi = 0;
    int rc;
    const bool pointwise = is_pointwise(s0.op);
    if (!pointwise && (rc = fill_stage(s0, p, 0)) != STRATA_OK) return rc;
    if (pointwise) {
        p.op = (int)s0.op;
        p.radius = 0;
    }
    // The tail: the tables in epi[], and, when it holds a chain step, the
    // whole tail as a step sequence naming the tables by index.
    bool seq = false;
    for (int i = 0; i < nstages; i++) seq = seq || stages[i].op == STRATA_OP_STEP;
    p.ninputs = 1;
    for (int i = pointwise ? 0 : 1; i < nstages; i++) {
        const strata_stage& s = stages[i];
        if (!is_pointwise(s.op) || s0.op == STRATA_OP_GRADIENT)
            return fail(STRATA_ENOTSUP,
                        "engine: a pipeline on the gpu backend is one stencil stage followed by pointwise stages");
        if (s.op == STRATA_OP_STEP) {
            if ((rc = fill_stage(s, p, 0)) != STRATA_OK) return rc;
            if (binary_step(s.kind)) {
                if (!pointwise)
                    return fail(STRATA_ENOTSUP,
                                "engine: a %s step reads a second input, which a stencil's pipeline on the gpu "
                                "backend does not take",
                                vec_name(s.kind));
                if (s.input + 1 > p.ninputs) p.ninputs = s.input + 1;
            }
            continue;
        }
        if ((rc = fill_stage(s, p, epi)) != STRATA_OK) return rc;
        if (seq) {
            if (p.nstep >= STRATA_MAX_STEPS)
                return fail(STRATA_EINVAL, "vec: chain has more than %d steps", STRATA_MAX_STEPS);
            p.step[p.nstep++] = strata::ChainStep{strata::kStepTable + epi, 0, 0.0f, 0.0f};
        }
        epi++;
    }
    p.nepi = epi;
    fold_tail(p);
    fold_slope_square(p);
    *nout = s0.op == STRATA_OP_GRADIENT ? 2 : 1;
    return STRATA_OK;
}

int check_operands(const strata_raster* src, int nsrc, const strata_raster* dst, int ndst, int nout, int r,
                   int nin = 1) {
    if (nsrc != nin || ndst != nout || !src || !dst)
        return fail(STRATA_EINVAL, "engine: kernel takes %d inputs and %d outputs, got %d and %d", nin, nout, nsrc,
                    ndst);
    int rc;
    for (int i = 0; i < ndst; i++) {
        if ((rc = validate("dst", i, dst[i])) != STRATA_OK) return rc;
        if (dst[i].width != dst[0].width || dst[i].height != dst[0].height)
            return fail(STRATA_EINVAL, "engine: dst[%d] is %lld×%lld, dst[0] is %lld×%lld", i, (long long)dst[i].width,
                        (long long)dst[i].height, (long long)dst[0].width, (long long)dst[0].height);
    }
    for (int j = 0; j < nsrc; j++) {
        if ((rc = validate("src", j, src[j])) != STRATA_OK) return rc;
        if (src[j].width != dst[0].width || src[j].height != dst[0].height)
            return fail(STRATA_EINVAL, "engine: src[%d] is %lld×%lld, dst[0] is %lld×%lld", j, (long long)src[j].width,
                        (long long)src[j].height, (long long)dst[0].width, (long long)dst[0].height);
        for (int i = 0; i < ndst; i++)
            if (src[j].valid && !dst[i].valid)
                return fail(STRATA_EINVAL,
                            "engine: an input has a validity mask but dst[%d].Valid is nil; allocate it with "
                            "raster.NewFloat32Like, or set Valid on its root raster before windowing",
                            i);
    }
    // A pointwise kernel's other inputs: each may be dst itself (read
    // before the cell is written), never a part of it at another offset.
    for (int j = 1; j < nsrc; j++)
        for (int i = 0; i < ndst; i++) {
            if (data_rel(dst[i], src[j]) == kPartial)
                return fail(STRATA_EINVAL, "engine: dst[%d] overlaps src[%d] at a different offset or stride", i, j);
            if (bits_rel(dst[i], src[j]) == kPartial)
                return fail(STRATA_EINVAL,
                            "engine: dst[%d] validity bits overlap src[%d]'s at a different offset or stride", i, j);
        }
    for (int i = 0; i < ndst; i++) {
        for (int j = i + 1; j < ndst; j++) {
            bool dm = r == 0 ? data_rel(dst[i], dst[j]) != kDisjoint : data_spans(dst[i], dst[j]);
            if (dm) return fail(STRATA_EINVAL, "engine: dst[%d] and dst[%d] share Data", i, j);
            bool bm = r == 0 ? bits_rel(dst[i], dst[j]) != kDisjoint : bit_spans(dst[i], dst[j]);
            if (bm) return fail(STRATA_EINVAL, "engine: dst[%d] and dst[%d] share validity bits", i, j);
        }
        const strata_raster& s = src[0];
        if (r > 0) {
            if (data_spans(dst[i], s))
                return fail(STRATA_EINVAL,
                            "engine: dst[%d] and src[0] share Data; a kernel with radius %d would read neighbours "
                            "it has already overwritten",
                            i, r);
            if (bit_spans(dst[i], s)) return fail(STRATA_EINVAL, "engine: dst[%d] and src[0] share validity bits", i);
            continue;
        }
        Relation d = data_rel(dst[i], s);
        if (d == kPartial)
            return fail(STRATA_EINVAL, "engine: dst[%d] overlaps src[0] at a different offset or stride", i);
        if (d == kSame && nout > 1)
            return fail(STRATA_EINVAL, "engine: dst[%d] is src[0]; only a kernel with one output runs in place", i);
        if (bits_rel(dst[i], s) == kPartial)
            return fail(STRATA_EINVAL,
                        "engine: dst[%d] validity bits overlap src[0]'s at a different offset or stride", i);
    }
    return STRATA_OK;
}

// A raster resolved to device memory.
struct DevOperand {
    float* data = nullptr;
    int64_t stride = 0;
    uint32_t* bits = nullptr;  // 32-bit view of the mask words
    int64_t bit_off = 0;       // bit of cell (0, 0) in bits
    int64_t lo_word = 0, hi_word = 0;  // 32-bit words holding the raster's bits
    // Host staging of the mask, for write-back.
    int64_t host_w0 = 0, nwords64 = 0;
};

// The 64-bit words [w0, w0 + n) that hold bits [off, off + cells).
void mask_words(int64_t off, int64_t cells, int64_t* w0, int64_t* n) {
    *w0 = off >> 6;
    *n = ((off + cells + 63) >> 6) - *w0;
}

// Page-locked room for the edge words of n destinations.
int ensure_edges(strata_ctx* c, size_t n) {
    if (c->n_edges >= 2 * n) return STRATA_OK;
    if (c->h_edges) cudaFreeHost(c->h_edges);
    c->h_edges = nullptr;
    c->n_edges = 0;
    const size_t want = std::max<size_t>(2 * n, 64);
    cudaError_t e = cudaHostAlloc(&c->h_edges, want * 8, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(e, "mask staging");
    c->n_edges = want;
    return STRATA_OK;
}

// Starts the copy of a host destination's mask back on stream s: the words
// wholly inside the raster's bit span straight into the caller's words,
// the first and last (which other rasters may share) into edge[0..1] for
// merge_edges once the stream is done.
cudaError_t mask_back(const strata_raster& r, const DevOperand& d, uint64_t* edge, cudaStream_t s) {
    const int64_t n = d.nwords64;
    const uint64_t* dev = reinterpret_cast<const uint64_t*>(d.bits);
    cudaError_t e = cudaSuccess;
    if (n > 2) e = cudaMemcpyAsync(r.valid + d.host_w0 + 1, dev + 1, (size_t)(n - 2) * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(edge, dev, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && n > 1) e = cudaMemcpyAsync(edge + 1, dev + n - 1, 8, cudaMemcpyDeviceToHost, s);
    return e;
}

// Merges the edge words mask_back fetched: only the raster's own bits of
// them change.
// Strips of one raster computed at once on several devices share their
// edge words, so the merges take turns.
std::mutex g_edge_mu;

void merge_edges(const strata_raster& r, const DevOperand& d, const uint64_t* edge) {
    std::lock_guard<std::mutex> lock(g_edge_mu);
    const int64_t lo = r.valid_offset, hi = r.valid_offset + span_cells(r);
    auto merge = [&](int64_t k, uint64_t v) {
        const int64_t w = d.host_w0 + k;
        uint64_t own = ~0ull;
        if (w * 64 < lo) own &= ~0ull << (lo - w * 64);
        if ((w + 1) * 64 > hi) own &= (hi - w * 64) >= 64 ? ~0ull : ((1ull << (hi - w * 64)) - 1);
        r.valid[w] = (r.valid[w] & ~own) | (v & own);
    };
    merge(0, edge[0]);
    if (d.nwords64 > 1) merge(d.nwords64 - 1, edge[1]);
}

// A destination's cells back to the host: one linear copy when its rows
// are contiguous, else a 2-D copy that leaves the gap cells alone.
cudaError_t data_back(const strata_raster& r, const DevOperand& d, cudaStream_t s) {
    if (r.stride == r.width)
        return cudaMemcpyAsync(r.data, d.data, (size_t)(r.width * r.height) * 4, cudaMemcpyDeviceToHost, s);
    return cudaMemcpy2DAsync(r.data, (size_t)r.stride * 4, d.data, (size_t)r.stride * 4, (size_t)r.width * 4,
                             (size_t)r.height, cudaMemcpyDeviceToHost, s);
}

int stage_in(strata_ctx* c, cudaStream_t st, const strata_raster& r, int slot, bool copy_data, DevOperand* d) {
    d->stride = r.stride;
    int64_t cells = span_cells(r);
    if (r.on_device) {
        d->data = r.data;
        if (r.valid) {
            int64_t w0 = (r.valid_offset >> 6);
            d->bits = reinterpret_cast<uint32_t*>(r.valid + w0);
            d->bit_off = r.valid_offset - w0 * 64;
        }
    } else {
        void* p;
        int rc = ensure(c, slot, (size_t)cells * 4, &p);
        if (rc) return rc;
        d->data = (float*)p;
        if (copy_data) {
            cudaError_t e = cudaMemcpyAsync(p, r.data, (size_t)cells * 4, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return cuda_fail(e, "copy to device");
        }
        if (r.valid) {
            int64_t w0, n;
            mask_words(r.valid_offset, cells, &w0, &n);
            void* m;
            if ((rc = ensure(c, slot + 1, (size_t)n * 8, &m))) return rc;
            cudaError_t e = cudaMemcpyAsync(m, r.valid + w0, (size_t)n * 8, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return cuda_fail(e, "copy mask to device");
            d->bits = (uint32_t*)m;
            d->bit_off = r.valid_offset - w0 * 64;
            d->host_w0 = w0;
            d->nwords64 = n;
        }
    }
    if (d->bits) {
        d->lo_word = d->bit_off >> 5;
        d->hi_word = (d->bit_off + cells - 1) >> 5;
    }
    return STRATA_OK;
}

// Copies a host destination back: its cells, and its mask bits merged into
// the caller's words (the first and last words may hold other rasters'
// bits).
int stage_out(strata_ctx* c, cudaStream_t st, const strata_raster& r, const DevOperand& d) {
    if (r.on_device) return STRATA_OK;
    cudaError_t e = data_back(r, d, st);
    if (e != cudaSuccess) return cuda_fail(e, "copy to host");
    if (r.valid) {
        int rc;
        if ((rc = ensure_edges(c, 1))) return rc;
        if ((e = mask_back(r, d, c->h_edges, st)) != cudaSuccess) return cuda_fail(e, "copy mask to host");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "copy mask to host");
        merge_edges(r, d, c->h_edges);
    }
    return STRATA_OK;
}

void fill_validity(ValidityParams& v, const DevOperand& s, bool src_masked, const DevOperand& d, int64_t dst_cells_span,
                   int64_t W, int64_t H, int r, int64_t y0, int64_t y1) {
    memset(&v, 0, sizeof v);
    if (src_masked) {
        v.src_bits = s.bits;
        v.src_off = s.bit_off;
        v.src_stride = s.stride;
        v.src_lo_word = s.lo_word;
        v.src_hi_word = s.hi_word;
    }
    v.dst_bits = d.bits;
    v.dst_off = d.bit_off;
    v.dst_stride = d.stride;
    v.out_x0 = 0;
    v.out_x1 = W;
    v.out_y0 = y0;
    v.out_y1 = y1;
    v.width = W;
    v.height = H;
    v.radius = r;
    // Words holding the region's bits: rows y0 .. y1-1.
    int64_t b0 = d.bit_off + y0 * d.stride;
    int64_t b1 = d.bit_off + (y1 - 1) * d.stride + W;  // exclusive
    (void)dst_cells_span;
    v.dst_lo_word = b0 >> 5;
    v.dst_words = ((b1 + 31) >> 5) - v.dst_lo_word;
}



// Wood's fit on the device (terrain/fit.go:111-170). Each raw fit sum is a
// separable correlation of the window: the column fold ColumnSum is the
// column correlation with unit taps (1·z is z exactly, so copying the first
// row and adding the rest gives the same bits), so p's sum is
// CorrelateSeparable with column taps 1 and row taps i, q's with column
// taps i and row taps 1, and curvature's r, s, t with (1, 3i²-r(r+1)),
// (i, i) and (3i²-r(r+1), 1): the separable kernels compute them in the
// reference's fold orders. The sums land in context scratch with the
// output's geometry, then the finishing pass scales them and applies the
// product (launch_fit_finish), and the validity kernel erodes the mask by
// the fit's radius.
int64_t launch_fit(strata_ctx* c, const LaunchParams& p, const ValidityParams* const v[2], cudaStream_t st,
                   int64_t* window) {
    const int r = p.fit;
    const int nd = p.op == STRATA_OP_CURVATURE ? 5 : 2;
    const int64_t ds = p.out_x1 - p.dst_x0, rows = p.out_y1 - p.dst_y0;
    float* d[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int i = 0; i < nd; i++) {
        void* q;
        if (ensure(c, kFitScratchSlot + i, (size_t)(rows * ds) * 4, &q)) return -2;
        d[i] = static_cast<float*>(q);
    }
    float ti[2 * STRATA_MAX_RADIUS + 1], t2[2 * STRATA_MAX_RADIUS + 1], ones[2 * STRATA_MAX_RADIUS + 1];
    for (int i = -r; i <= r; i++) {
        ti[i + r] = (float)i;
        t2[i + r] = (float)(3 * i * i - r * (r + 1));
        ones[i + r] = 1.0f;
    }
    // (column taps, row taps) of p, q, r, s, t
    const float* taps[5][2] = {{ones, ti}, {ti, ones}, {ones, t2}, {ti, ti}, {t2, ones}};
    int64_t blocks = 0, cells = 0;
    for (int i = 0; i < nd; i++) {
        LaunchParams q = p;
        q.op = STRATA_OP_SEPARABLE;
        q.kind = 0;
        q.fit = 0;
        q.nepi = 0;
        q.nstep = 0;
        memset(&q.vf, 0, sizeof q.vf);
        for (int j = 0; j <= 2 * r; j++) {
            q.w[j] = taps[i][1][j];
            q.w[17 + j] = taps[i][0][j];
        }
        q.dst0 = d[i];
        q.dst0_stride = ds;
        q.dst1 = nullptr;
        int64_t wc = 0;
        const int64_t t = strata::launch_data(q, st, &wc);
        if (t < 0) return -1;
        blocks += t;
        cells += wc;
    }
    strata::launch_fit_finish(p, d, ds, st);
    for (int i = 0; i < 2; i++)
        if (v[i]) strata::launch_validity(*v[i], st);
    if (window) *window = cells;
    return blocks;
}

// The failure-path test's switch (STRATA_TEST_STALL_FIRST_WAIT=1): the TMA
// march then reports a bounded wait that ran out, with nothing faulted.
bool test_stall_requested() {
    const char* v = getenv("STRATA_TEST_STALL_FIRST_WAIT");
    return v && v[0] == '1';
}

}  // namespace

extern "C" int strata_process(strata_ctx* c, const strata_stage* stages, int nstages, const strata_raster* src,
                              int nsrc, const strata_raster* dst, int ndst, const strata_exec_opts* opts,
                              strata_stats* stats) {
    if (!c) return fail(STRATA_EINVAL, "engine: nil context");
    LaunchParams p;
    int nout = 0;
    int rc = plan_stages(stages, nstages, p, &nout);
    if (rc) return rc;
    if ((rc = check_opts(opts))) return rc;
    // A pointwise pipeline reads every input it is given (vec.Chain.Run
    // checks the ones it never reads too), at least those its steps name.
    const bool chain = is_pointwise((uint32_t)p.op);
    const int nin = chain && nsrc >= p.ninputs && nsrc <= STRATA_MAX_INPUTS ? nsrc : p.ninputs;
    if ((rc = check_operands(src, nsrc, dst, ndst, nout, p.radius, nin))) return rc;
    p.ninputs = nin;

    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard device_guard(c->device);
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    const int64_t W = src[0].width, H = src[0].height;

    DevOperand ds, dd[2], dx[STRATA_MAX_INPUTS];
    if ((rc = stage_in(c, st, src[0], 0, true, &ds))) return rc;
    for (int j = 1; j < nin; j++)
        if ((rc = stage_in(c, st, src[j], kInputSlot + 2 * j, true, &dx[j]))) return rc;
    dx[0] = ds;
    for (int i = 0; i < ndst; i++)
        if ((rc = stage_in(c, st, dst[i], 2 + 2 * i, false, &dd[i]))) return rc;

    for (int j = 0; j < nin; j++) {
        p.in[j] = dx[j].data;
        p.in_stride[j] = dx[j].stride;
    }
    p.src = ds.data;
    p.src_stride = ds.stride;
    p.src_x0 = p.src_y0 = 0;
    p.src_w = W;
    p.src_h = H;
    p.dst0 = dd[0].data;
    p.dst0_stride = dd[0].stride;
    if (ndst > 1) {
        p.dst1 = dd[1].data;
        p.dst1_stride = dd[1].stride;
    }
    p.dst_x0 = p.dst_y0 = 0;
    p.width = W;
    p.height = H;
    p.out_x0 = 0;
    p.out_x1 = W;
    p.status = c->d_status;
    p.test_stall = test_stall_requested();

    // Row strips: the whole raster at once, or strips of about 2^22 cells
    // with the cancel flag polled between them.
    const volatile int32_t* cancel = opts ? opts->cancel : nullptr;
    int64_t strip = H;
    if (cancel) {
        strip = ((int64_t)1 << 22) / W;
        strip = (strip + 31) / 32 * 32;
        if (strip < 32) strip = 32;
    }
    int64_t bands = 0, window = 0, done_rows = 0;
    bool canceled = false;
    for (int64_t y0 = 0; y0 < H; y0 += strip) {
        if (cancel && *cancel) {
            canceled = true;
            break;
        }
        int64_t y1 = y0 + strip < H ? y0 + strip : H;
        p.out_y0 = y0;
        p.out_y1 = y1;
        int64_t wc = 0;
        ValidityParams vp[2];
        const ValidityParams* vs[2] = {nullptr, nullptr};
        for (int i = 0; i < ndst && nin == 1; i++) {
            if (!dst[i].valid) continue;
            fill_validity(vp[i], ds, src[0].valid != nullptr, dd[i], span_cells(dst[i]), W, H, p.radius, y0, y1);
            vs[i] = &vp[i];
        }
        int64_t t = p.fit ? launch_fit(c, p, vs, st, &wc) : strata::launch_stage(p, vs, st, &wc);
        if (t >= 0 && nin > 1 && dst[0].valid) {
            strata::AndValidityParams av;
            memset(&av, 0, sizeof av);
            for (int j = 0; j < nin; j++) {
                av.src_bits[j] = src[j].valid ? dx[j].bits : nullptr;
                av.src_off[j] = dx[j].bit_off;
                av.src_stride[j] = dx[j].stride;
            }
            av.nsrc = nin;
            av.dst_bits = dd[0].bits;
            av.dst_off = dd[0].bit_off;
            av.dst_stride = dd[0].stride;
            av.width = W;
            av.y0 = y0;
            av.y1 = y1;
            strata::launch_and_validity(av, st);
        }
        if (t == -2) return fail(STRATA_ENOMEM, "engine: no device memory for the fit's sums");
        if (t < 0) return fail(STRATA_ENOTSUP, "engine: op %d at radius %d has no device kernel", p.op, p.radius);
        bands += t;
        window += wc;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
        if (cancel) {
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_fail(e, "kernel");
        }
        done_rows = y1;
    }
    bool all_device = src[0].on_device && dst[0].on_device && (ndst < 2 || dst[1].on_device);
    for (int i = 0; i < ndst; i++)
        if ((rc = stage_out(c, st, dst[i], dd[i]))) return rc;
    if (!(all_device && opts && (opts->flags & STRATA_EXEC_ASYNC))) {
        if ((rc = take_status(c, st))) return rc;
    }
    if (stats) {
        int64_t cells = done_rows * W;
        stats->cells += cells;
        stats->ideal += cells * 4 * (nin + nout);
        stats->bands += bands;
        stats->kernel_read += window * 4;
        stats->kernel_written += cells * 4 * nout;
    }
    if (canceled) return fail(STRATA_ECANCELED, "context canceled");
    return STRATA_OK;
}

// ---------------------------------------------------------------------------
// Row strips of one raster (the multi-GPU split): a strip's outputs are
// the rows strata_process writes for them over the whole raster.

extern "C" int strata_process_strip(strata_ctx* c, const strata_stage* stages, int nstages, const strata_raster* src,
                                    const strata_raster* dst, int ndst, const strata_strip* strip,
                                    const strata_exec_opts* opts, strata_stats* stats) {
    if (!c) return fail(STRATA_EINVAL, "engine: nil context");
    if (!strip || !src || !dst) return fail(STRATA_EINVAL, "engine: nil strip operands");
    LaunchParams p;
    int nout = 0;
    int rc = plan_stages(stages, nstages, p, &nout);
    if (rc) return rc;
    if ((rc = check_opts(opts))) return rc;
    if (p.ninputs > 1) return fail(STRATA_ENOTSUP, "engine: a chain over several inputs has no strip form");
    if (ndst != nout)
        return fail(STRATA_EINVAL, "engine: kernel takes 1 inputs and %d outputs, got 1 and %d", nout, ndst);
    if ((rc = validate("src", 0, src[0]))) return rc;
    for (int i = 0; i < ndst; i++) {
        if ((rc = validate("dst", i, dst[i]))) return rc;
        if (dst[i].width != src[0].width || dst[i].height != dst[0].height)
            return fail(STRATA_EINVAL, "engine: dst[%d] is %lld×%lld, the strip is %lld×%lld", i,
                        (long long)dst[i].width, (long long)dst[i].height, (long long)src[0].width,
                        (long long)dst[0].height);
        if (src[0].valid && !dst[i].valid)
            return fail(STRATA_EINVAL,
                        "engine: an input has a validity mask but dst[%d].Valid is nil; allocate it with "
                        "raster.NewFloat32Like, or set Valid on its root raster before windowing",
                        i);
        if (p.radius > 0 && (data_spans(dst[i], src[0]) || bit_spans(dst[i], src[0])))
            return fail(STRATA_EINVAL, "engine: dst[%d] and src[0] share memory; a kernel with radius %d would read "
                                       "neighbours it has already overwritten", i, p.radius);
        for (int j = 0; j < i; j++)
            if (data_spans(dst[i], dst[j]) || bit_spans(dst[i], dst[j]))
                return fail(STRATA_EINVAL, "engine: dst[%d] and dst[%d] share memory", j, i);
    }
    const int64_t H = strip->height, W = src[0].width;
    const int64_t s0 = strip->src_row, s1 = s0 + src[0].height;
    const int64_t y0 = strip->dst_row, y1 = y0 + dst[0].height;
    const int r = p.radius;
    if (y0 < 0 || y1 > H || s0 < 0 || s1 > H)
        return fail(STRATA_EINVAL, "engine: strip rows [%lld, %lld) and source rows [%lld, %lld) must lie in the "
                                   "raster's %lld rows",
                    (long long)y0, (long long)y1, (long long)s0, (long long)s1, (long long)H);
    if (s0 > std::max<int64_t>(0, y0 - r) || s1 < std::min<int64_t>(H, y1 + r))
        return fail(STRATA_EINVAL, "engine: source rows [%lld, %lld) do not cover rows [%lld, %lld) that output rows "
                                   "[%lld, %lld) read at radius %d",
                    (long long)s0, (long long)s1, (long long)std::max<int64_t>(0, y0 - r),
                    (long long)std::min<int64_t>(H, y1 + r), (long long)y0, (long long)y1, r);

    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard device_guard(c->device);
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    DevOperand ds, dd[2];
    if ((rc = stage_in(c, st, src[0], 0, true, &ds))) return rc;
    for (int i = 0; i < ndst; i++)
        if ((rc = stage_in(c, st, dst[i], 2 + 2 * i, false, &dd[i]))) return rc;
    p.src = ds.data;
    p.src_stride = ds.stride;
    p.src_x0 = 0;
    p.src_y0 = s0;
    p.src_w = W;
    p.src_h = s1 - s0;
    p.in[0] = ds.data;
    p.in_stride[0] = ds.stride;
    p.dst0 = dd[0].data;
    p.dst0_stride = dd[0].stride;
    if (ndst > 1) {
        p.dst1 = dd[1].data;
        p.dst1_stride = dd[1].stride;
    }
    p.dst_x0 = 0;
    p.dst_y0 = y0;
    p.width = W;
    p.height = H;
    p.out_x0 = 0;
    p.out_x1 = W;
    p.out_y0 = y0;
    p.out_y1 = y1;
    p.status = c->d_status;
    p.test_stall = test_stall_requested();
    ValidityParams vp[2];
    const ValidityParams* vs[2] = {nullptr, nullptr};
    for (int i = 0; i < ndst; i++) {
        if (!dst[i].valid) continue;
        ValidityParams& v = vp[i];
        memset(&v, 0, sizeof v);
        if (src[0].valid) {
            v.src_bits = ds.bits;
            v.src_off = ds.bit_off;
            v.src_stride = ds.stride;
            v.src_lo_word = ds.lo_word;
            v.src_hi_word = ds.hi_word;
        }
        v.src_y0 = s0;
        v.dst_bits = dd[i].bits;
        v.dst_off = dd[i].bit_off;
        v.dst_stride = dd[i].stride;
        v.dst_y0 = y0;
        v.out_x1 = W;
        v.out_y0 = y0;
        v.out_y1 = y1;
        v.width = W;
        v.height = H;
        v.radius = r;
        const int64_t b0 = dd[i].bit_off, b1 = dd[i].bit_off + (y1 - y0 - 1) * dd[i].stride + W;
        v.dst_lo_word = b0 >> 5;
        v.dst_words = ((b1 + 31) >> 5) - v.dst_lo_word;
        vs[i] = &v;
    }
    int64_t wc = 0;
    const int64_t t = p.fit ? launch_fit(c, p, vs, st, &wc) : strata::launch_stage(p, vs, st, &wc);
    if (t == -2) return fail(STRATA_ENOMEM, "engine: no device memory for the fit's sums");
    if (t < 0) return fail(STRATA_ENOTSUP, "engine: op %d at radius %d has no device kernel", p.op, p.radius);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    for (int i = 0; i < ndst; i++)
        if ((rc = stage_out(c, st, dst[i], dd[i]))) return rc;
    const bool all_device = src[0].on_device && dst[0].on_device && (ndst < 2 || dst[1].on_device);
    if (!(all_device && opts && (opts->flags & STRATA_EXEC_ASYNC)))
        if ((rc = take_status(c, st))) return rc;
    if (stats) {
        const int64_t cells = (y1 - y0) * W;
        stats->cells += cells;
        stats->ideal += cells * 4 * (1 + nout);
        stats->bands += t;
        stats->kernel_read += wc * 4;
        stats->kernel_written += cells * 4 * nout;
    }
    return STRATA_OK;
}

// A view of rows [y0, y1) of r.
static strata_raster rows_of(const strata_raster& r, int64_t y0, int64_t y1) {
    strata_raster v = r;
    v.data = r.data + y0 * r.stride;
    v.height = y1 - y0;
    if (r.valid) v.valid_offset = r.valid_offset + y0 * r.stride;
    return v;
}

extern "C" int strata_process_multi(strata_ctx* const* ctxs, int nctx, const strata_stage* stages, int nstages,
                                    const strata_raster* src, int nsrc, const strata_raster* dst, int ndst,
                                    const strata_exec_opts* opts, strata_stats* stats) {
    if (!ctxs || nctx < 1) return fail(STRATA_EINVAL, "engine: no devices");
    for (int i = 0; i < nctx; i++)
        if (!ctxs[i]) return fail(STRATA_EINVAL, "engine: nil context %d", i);
    if (nctx == 1) return strata_process(ctxs[0], stages, nstages, src, nsrc, dst, ndst, opts, stats);
    LaunchParams p;
    int nout = 0;
    int rc = plan_stages(stages, nstages, p, &nout);
    if (rc) return rc;
    if ((rc = check_opts(opts))) return rc;
    if (p.ninputs > 1 || nsrc > 1)
        return fail(STRATA_ENOTSUP, "engine: a chain over several inputs has no multi-device form");
    if ((rc = check_operands(src, nsrc, dst, ndst, nout, p.radius))) return rc;
    if (opts && (opts->stream || opts->cancel))
        return fail(STRATA_EINVAL, "engine: a multi-device call takes no stream or cancel flag");
    if (src[0].on_device || dst[0].on_device || (ndst > 1 && dst[1].on_device))
        return fail(STRATA_ENOTSUP, "engine: a multi-device call takes host rasters");
    // shard.strips: contiguous output rows, as equal as can be, each with
    // its halo rows read from the host by its own device.
    const int64_t H = src[0].height, r = p.radius;
    const int64_t base = H / nctx, extra = H % nctx;
    std::vector<int> codes((size_t)nctx, STRATA_OK);
    std::vector<std::string> errs((size_t)nctx);
    std::vector<strata_stats> part((size_t)nctx);
    std::vector<std::thread> threads;
    int64_t y = 0;
    for (int i = 0; i < nctx; i++) {
        const int64_t n = base + (i < extra ? 1 : 0);
        const int64_t y0 = y, y1 = y + n;
        y = y1;
        if (n == 0) continue;
        threads.emplace_back([&, i, y0, y1]() {
            const int64_t s0 = std::max<int64_t>(0, y0 - r), s1 = std::min<int64_t>(H, y1 + r);
            const strata_raster sv = rows_of(src[0], s0, s1);
            strata_raster dv[2];
            for (int k = 0; k < ndst; k++) dv[k] = rows_of(dst[k], y0, y1);
            const strata_strip strip = {H, s0, y0};
            memset(&part[(size_t)i], 0, sizeof(strata_stats));
            codes[(size_t)i] = strata_process_strip(ctxs[i], stages, nstages, &sv, dv, ndst, &strip, opts,
                                                    &part[(size_t)i]);
            if (codes[(size_t)i] != STRATA_OK) errs[(size_t)i] = g_err;
        });
    }
    for (auto& t : threads) t.join();
    for (int i = 0; i < nctx; i++)
        if (codes[(size_t)i] != STRATA_OK) {
            g_err = errs[(size_t)i];
            return codes[(size_t)i];
        }
    if (stats)
        for (const strata_stats& q : part) {
            stats->cells += q.cells;
            stats->ideal += q.ideal;
            stats->bands += q.bands;
            stats->kernel_read += q.kernel_read;
            stats->kernel_written += q.kernel_written;
        }
    return STRATA_OK;
}

// ---------------------------------------------------------------------------
// Stage builders.

namespace {

void stage_init(strata_stage* s, uint32_t op) {
    memset(s, 0, sizeof *s);
    s->op = op;
}

// terrain.resolveCells (terrain/stencil.go:16-34).
int resolve_cells(double cs, double csy, double z, double* cx, double* cy, double* zf) {
    if (!(cs > 0) || std::isinf(cs))
        return fail(STRATA_EINVAL, "terrain: CellSize must be positive and finite, got %s", fmt_v(cs).c_str());
    if (csy == 0) csy = cs;
    if (!(csy > 0) || std::isinf(csy))
        return fail(STRATA_EINVAL, "terrain: CellSizeY must be positive and finite (or 0 for CellSize), got %s",
                    fmt_v(csy).c_str());
    if (z == 0) z = 1;
    if (std::isnan(z) || std::isinf(z))
        return fail(STRATA_EINVAL, "terrain: ZFactor must be finite, got %s", fmt_v(z).c_str());
    *cx = cs;
    *cy = csy;
    *zf = z;
    return STRATA_OK;
}

bool usable(float k) { return k != 0 && !std::isinf(k); }

// terrain.cellSizes (terrain/stencil.go:37-49) with stencil.HornScales
// (internal/stencil/horn.go:114-116).
int horn_scales(double cs, double csy, double z, float* kx, float* ky) {
    double cx, cy, zf;
    int rc = resolve_cells(cs, csy, z, &cx, &cy, &zf);
    if (rc) return rc;
    *kx = (float)(zf / (8 * cx));
    *ky = (float)(zf / (8 * cy));
    if (!usable(*kx) || !usable(*ky))
        return fail(STRATA_EINVAL,
                    "terrain: ZFactor/(8·CellSize) and ZFactor/(8·CellSizeY) must be finite and non-zero as float32, "
                    "got %s and %s for CellSize %s, CellSizeY %s and ZFactor %s",
                    fmt_v(*kx, true).c_str(), fmt_v(*ky, true).c_str(), fmt_v(cs).c_str(), fmt_v(csy).c_str(),
                    fmt_v(z).c_str());
    return STRATA_OK;
}

// The fit-radius switch of terrain/fit.go:187-226: 0 is Horn's 3x3
// kernel, 1..8 Wood's fit (checked at terrain/fit.go:37-40).
int fit_radius(int32_t fr) {
    if (fr < 0 || fr > STRATA_MAX_RADIUS)
        return fail(STRATA_EINVAL, "terrain: FitRadius must be 0 to %d, got %d", STRATA_MAX_RADIUS, fr);
    return STRATA_OK;
}

// newWoodFit (terrain/fit.go:38-66): the fit's factors kp, kq, kr, kt, ks,
// each computed in float64 and rounded once.
int wood_fit(int r, double cs, double csy, double zf, float* k) {
    double cx, cy, z;
    int rc = resolve_cells(cs, csy, zf, &cx, &cy, &z);
    if (rc) return rc;
    double q = 0;
    for (int i = -r; i <= r; i++) {
        const double w = 3.0 * i * i - r * (r + 1);
        q += w * w;
    }
    const double kk = 2 * r + 1, s = (double)(r * (r + 1) * (2 * r + 1)) / 3;
    k[0] = (float)(z / (kk * s * cx));
    k[1] = (float)(z / (kk * s * cy));
    k[2] = (float)(6 * z / (kk * q * cx * cx));
    k[3] = (float)(6 * z / (kk * q * cy * cy));
    k[4] = (float)(z / (s * s * cx * cy));
    for (int i = 0; i < 5; i++)
        if (!usable(k[i]))
            return fail(STRATA_EINVAL,
                        "terrain: the quadratic fit's factors ZFactor/(K·S·CellSize), 6·ZFactor/(K·Q·CellSize²) and "
                        "ZFactor/(S²·CellSize·CellSizeY), and the same for CellSizeY, must be finite and non-zero as "
                        "float32, got %s, %s, %s, %s and %s for CellSize %s, CellSizeY %s, ZFactor %s and FitRadius %d",
                        fmt_v(k[0], true).c_str(), fmt_v(k[1], true).c_str(), fmt_v(k[2], true).c_str(),
                        fmt_v(k[3], true).c_str(), fmt_v(k[4], true).c_str(), fmt_v(cs).c_str(), fmt_v(csy).c_str(),
                        fmt_v(zf).c_str(), r);
    return STRATA_OK;
}

// The derivative part of a terrain stage: Horn's 3x3 scales (kx, ky in
// k[0..1], radius 1) when fr is 0, else Wood's fit (fit_stage); *base is
// where the product's constants go (2 for Horn, 5 for the fit).
int fit_stage(uint32_t op, int r, double cs, double csy, double z, strata_stage* out);
int deriv_stage(uint32_t op, int fr, double cs, double csy, double z, strata_stage* out, int* base) {
    if (fr) {
        *base = 5;
        return fit_stage(op, fr, cs, csy, z, out);
    }
    float kx, ky;
    int rc = horn_scales(cs, csy, z, &kx, &ky);
    if (rc) return rc;
    stage_init(out, op);
    out->radius = 1;
    out->k[0] = kx;
    out->k[1] = ky;
    *base = 2;
    return STRATA_OK;
}

// A product of Wood's fit (terrain/fit.go:187-226): the op, the fit's
// radius and factors; the caller adds the product's constants from k[5].
int fit_stage(uint32_t op, int r, double cs, double csy, double z, strata_stage* out) {
    float k[5];
    int rc = wood_fit(r, cs, csy, z, k);
    if (rc) return rc;
    stage_init(out, op);
    out->radius = r;
    out->flags = STRATA_STAGE_FIT;
    for (int i = 0; i < 5; i++) out->k[i] = k[i];
    return STRATA_OK;
}

int check_focal_radius(int r) {
    if (r < 1 || r > STRATA_MAX_RADIUS)
        return fail(STRATA_EINVAL, "focal: Radius must be 1 to %d, got %d", STRATA_MAX_RADIUS, r);
    return STRATA_OK;
}

int check_finite(const char* what, const float* v, int n) {
    for (int i = 0; i < n; i++)
        if (!finite32(v[i]))
            return fail(STRATA_EINVAL, "focal: %s must be finite, got %s at index %d", what, fmt_v(v[i], true).c_str(),
                        i);
    return STRATA_OK;
}

// transfer.checkIncreasing (transfer/transfer.go:225-239).
int check_increasing(const char* op, const char* name, const float* xs, int n) {
    for (int i = 0; i < n; i++)
        if (xs[i] != xs[i]) return fail(STRATA_EINVAL, "%s: %s must not hold NaN, but %s[%d] is NaN", op, name, name, i);
    for (int i = 1; i < n; i++)
        if (!(xs[i - 1] < xs[i]))
            return fail(STRATA_EINVAL, "%s: %s must be strictly increasing, but %s[%d] = %s is not above %s[%d] = %s", op,
                        name, name, i, fmt_v(xs[i], true).c_str(), name, i - 1, fmt_v(xs[i - 1], true).c_str());
    return STRATA_OK;
}

}  // namespace

extern "C" int strata_stage_gradient(const strata_gradient_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    int rc = fit_radius(o->fit_radius);
    if (rc) return rc;
    if (o->fit_radius)
        return fit_stage(STRATA_OP_GRADIENT, o->fit_radius, o->cell_size, o->cell_size_y, o->z_factor, out);
    float kx, ky;
    if ((rc = horn_scales(o->cell_size, o->cell_size_y, o->z_factor, &kx, &ky))) return rc;
    stage_init(out, STRATA_OP_GRADIENT);
    out->radius = 1;
    out->k[0] = kx;
    out->k[1] = ky;
    return STRATA_OK;
}

extern "C" int strata_stage_slope(const strata_slope_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    int rc = fit_radius(o->fit_radius);
    if (rc) return rc;
    int base;
    if ((rc = deriv_stage(STRATA_OP_SLOPE, o->fit_radius, o->cell_size, o->cell_size_y, o->z_factor, out, &base)))
        return rc;
    // terrain.slopeScale (terrain/slope.go:84-95).
    float scale;
    int take_atan;
    switch (o->units) {
    case 0: scale = (float)(180 / M_PI); take_atan = 1; break;
    case 2: scale = 1; take_atan = 1; break;
    case 1: scale = 100; take_atan = 0; break;
    default: return fail(STRATA_EINVAL, "terrain: unknown SlopeUnits %d", o->units);
    }
    out->kind = take_atan;
    out->k[base] = scale;
    return STRATA_OK;
}

extern "C" int strata_stage_aspect(const strata_aspect_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    int rc = fit_radius(o->fit_radius);
    if (rc) return rc;
    int base;
    if ((rc = deriv_stage(STRATA_OP_ASPECT, o->fit_radius, o->cell_size, o->cell_size_y, o->z_factor, out, &base)))
        return rc;
    out->kind = o->trigonometric ? 1 : 0;
    out->k[base] = o->zero_for_flat ? 0.0f : -1.0f;  // terrain.aspectFlat, AspectFlat = -1
    return STRATA_OK;
}

extern "C" int strata_stage_hillshade(const strata_hillshade_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    int rc = fit_radius(o->fit_radius);
    if (rc) return rc;
    int base;
    if ((rc = deriv_stage(STRATA_OP_HILLSHADE, o->fit_radius, o->cell_size, o->cell_size_y, o->z_factor, out,
                          &base)))
        return rc;
    // terrain.hillshadeLight (terrain/hillshade.go:94-117).
    double az = o->azimuth, alt = o->altitude;
    if (std::isnan(az) || std::isinf(az))
        return fail(STRATA_EINVAL, "terrain: Azimuth must be finite, got %s", fmt_v(az).c_str());
    if (az == 0) az = 315;
    if (alt == 0) alt = 45;
    if (!(alt > 0 && alt <= 90))
        return fail(STRATA_EINVAL, "terrain: Altitude must be in (0, 90] (or 0 for 45), got %s",
                    fmt_v(o->altitude).c_str());
    az = std::fmod(az, 360);
    az = az * M_PI / 180;
    alt = alt * M_PI / 180;
    out->k[base] = (float)(255 * std::sin(alt));
    out->k[base + 1] = (float)(-255 * std::cos(alt) * std::sin(az));
    out->k[base + 2] = (float)(255 * std::cos(alt) * std::cos(az));
    return STRATA_OK;
}

extern "C" int strata_stage_curvature(const strata_curvature_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    int rc = fit_radius(o->fit_radius);
    if (rc) return rc;
    if (o->fit_radius) {
        if ((rc = fit_stage(STRATA_OP_CURVATURE, o->fit_radius, o->cell_size, o->cell_size_y, o->z_factor, out)))
            return rc;
        if (o->type < 0 || o->type > 2) return fail(STRATA_EINVAL, "terrain: unknown CurvatureType %d", o->type);
        out->kind = o->type;
        return STRATA_OK;
    }
    double cx, cy, z;
    if ((rc = resolve_cells(o->cell_size, o->cell_size_y, o->z_factor, &cx, &cy, &z))) return rc;
    if (o->type < 0 || o->type > 2) return fail(STRATA_EINVAL, "terrain: unknown CurvatureType %d", o->type);
    // stencil.ZTScales (internal/stencil/curvature.go:29-33).
    float k[5] = {(float)(z / (2 * cx)), (float)(z / (2 * cy)), (float)(z / (cx * cx)), (float)(z / (cy * cy)),
                  (float)(z / (4 * cx * cy))};
    for (float v : k)
        if (!usable(v))
            return fail(STRATA_EINVAL,
                        "terrain: ZFactor/(2·CellSize), ZFactor/CellSize² and ZFactor/(4·CellSize·CellSizeY), and the "
                        "same for CellSizeY, must be finite and non-zero as float32, got %s, %s, %s, %s and %s for "
                        "CellSize %s, CellSizeY %s and ZFactor %s",
                        fmt_v(k[0], true).c_str(), fmt_v(k[1], true).c_str(), fmt_v(k[2], true).c_str(),
                        fmt_v(k[3], true).c_str(), fmt_v(k[4], true).c_str(), fmt_v(o->cell_size).c_str(),
                        fmt_v(o->cell_size_y).c_str(), fmt_v(o->z_factor).c_str());
    stage_init(out, STRATA_OP_CURVATURE);
    out->radius = 1;
    out->kind = o->type;
    for (int i = 0; i < 5; i++) out->k[i] = k[i];
    return STRATA_OK;
}

extern "C" int strata_stage_ruggedness(const strata_ruggedness_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    int r = o->radius == 0 ? 1 : o->radius;
    if (r < 1 || r > STRATA_MAX_RADIUS)
        return fail(STRATA_EINVAL, "terrain: RuggednessOptions.Radius must be 0 to %d, got %d", STRATA_MAX_RADIUS,
                    o->radius);
    if (o->type < 0 || o->type > 3) return fail(STRATA_EINVAL, "terrain: unknown RuggednessType %d", o->type);
    stage_init(out, STRATA_OP_RUGGEDNESS);
    out->radius = r;
    out->kind = o->type;
    return STRATA_OK;
}

extern "C" int strata_stage_correlate(const strata_weights_options* o, int convolve, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "focal: nil options");
    int rc = check_focal_radius(o->radius);
    if (rc) return rc;
    int d = 2 * o->radius + 1;
    if (o->nweights != d * d || (!o->weights && o->nweights))
        return fail(STRATA_EINVAL, "focal: Radius %d needs %d×%d = %d Weights, got %d", o->radius, d, d, d * d,
                    o->nweights);
    if ((rc = check_finite("Weights", o->weights, o->nweights))) return rc;
    stage_init(out, STRATA_OP_CORRELATE);
    out->radius = o->radius;
    out->flags = convolve ? STRATA_STAGE_ROTATE180 : 0;
    out->table[0] = o->weights;
    out->table_len[0] = o->nweights;
    return STRATA_OK;
}

extern "C" int strata_stage_separable(const strata_separable_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "focal: nil options");
    int rc = check_focal_radius(o->radius);
    if (rc) return rc;
    int d = 2 * o->radius + 1;
    if (o->nrow != d || o->ncol != d || !o->row || !o->col)
        return fail(STRATA_EINVAL, "focal: Radius %d needs %d Row and %d Col taps, got %d and %d", o->radius, d, d,
                    o->nrow, o->ncol);
    if ((rc = check_finite("Row taps", o->row, o->nrow))) return rc;
    if ((rc = check_finite("Col taps", o->col, o->ncol))) return rc;
    stage_init(out, STRATA_OP_SEPARABLE);
    out->radius = o->radius;
    out->table[0] = o->row;
    out->table_len[0] = o->nrow;
    out->table[1] = o->col;
    out->table_len[1] = o->ncol;
    return STRATA_OK;
}

extern "C" int strata_stage_box(const strata_box_options* o, uint32_t op, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "focal: nil options");
    if (op != STRATA_OP_MEAN && op != STRATA_OP_MIN && op != STRATA_OP_MAX)
        return fail(STRATA_EINVAL, "focal: op %u is not Mean, Min or Max", op);
    int rc = check_focal_radius(o->radius);
    if (rc) return rc;
    stage_init(out, op);
    out->radius = o->radius;
    return STRATA_OK;
}

extern "C" int strata_stage_lookup(const float* xs, const float* ys, int32_t n, strata_stage* out) {
    const char* op = "transfer.Lookup";
    if (!out) return fail(STRATA_EINVAL, "%s: nil stage", op);
    if (n < 0) return fail(STRATA_EINVAL, "%s: negative table length %d", op, n);
    if (n == 0) return fail(STRATA_EINVAL, "%s: the table needs at least one knot", op);
    int rc = check_increasing(op, "xs", xs, n);
    if (rc) return rc;
    for (int i = 0; i < n; i++)
        if (!finite32(xs[i]))
            return fail(STRATA_EINVAL, "%s: xs must be finite, but xs[%d] = %s", op, i, fmt_v(xs[i], true).c_str());
    if (n > STRATA_MAX_KNOTS)
        return fail(STRATA_ENOTSUP, "%s: the gpu backend takes at most %d knots, got %d", op, STRATA_MAX_KNOTS, n);
    stage_init(out, STRATA_OP_LOOKUP);
    out->table[0] = xs;
    out->table[1] = ys;
    out->table_len[0] = n;
    out->table_len[1] = n;
    return STRATA_OK;
}

extern "C" int strata_stage_reclass(const float* breaks, int32_t nbreaks, const float* values, int32_t nvalues,
                                    strata_stage* out) {
    const char* op = "transfer.Reclass";
    if (!out) return fail(STRATA_EINVAL, "%s: nil stage", op);
    if (nvalues != nbreaks + 1)
        return fail(STRATA_EINVAL, "%s: values must hold one more element than breaks, got %d values and %d breaks", op,
                    nvalues, nbreaks);
    int rc = check_increasing(op, "breaks", breaks, nbreaks);
    if (rc) return rc;
    if (nbreaks > STRATA_MAX_KNOTS)
        return fail(STRATA_ENOTSUP, "%s: the gpu backend takes at most %d breaks, got %d", op, STRATA_MAX_KNOTS,
                    nbreaks);
    stage_init(out, STRATA_OP_RECLASS);
    out->table[0] = breaks;
    out->table[1] = values;
    out->table_len[0] = nbreaks;
    out->table_len[1] = nvalues;
    return STRATA_OK;
}

extern "C" int strata_stage_step(int32_t op, int32_t input, float k0, float k1, strata_stage* out) {
    if (!out) return fail(STRATA_EINVAL, "vec: nil stage");
    int rc = check_step(op, input);
    if (rc) return rc;
    stage_init(out, STRATA_OP_STEP);
    out->kind = op;
    out->input = input;
    out->k[0] = k0;
    out->k[1] = k1;
    return STRATA_OK;
}

extern "C" int strata_stage_rescale(float a, float b, strata_stage* out) {
    return strata_stage_step(STRATA_VEC_AFFINE, -1, a, b, out);
}

// transfer.rescaleCoeffs (transfer/transfer.go:236-250).
extern "C" int strata_stage_rescale_range(float in_lo, float in_hi, float out_lo, float out_hi, strata_stage* out) {
    const char* op = "transfer.RescaleRange";
    if (!out) return fail(STRATA_EINVAL, "%s: nil stage", op);
    if (!finite32(in_lo) || !finite32(in_hi) || in_lo == in_hi)
        return fail(STRATA_EINVAL, "%s: inLo and inHi must be finite and different, got %s and %s", op,
                    fmt_v(in_lo, true).c_str(), fmt_v(in_hi, true).c_str());
    if (!finite32(out_lo) || !finite32(out_hi))
        return fail(STRATA_EINVAL, "%s: outLo and outHi must be finite, got %s and %s", op, fmt_v(out_lo, true).c_str(),
                    fmt_v(out_hi, true).c_str());
    const float a = (float)(((double)out_hi - (double)out_lo) / ((double)in_hi - (double)in_lo));
    const float b = (float)((double)out_lo - (double)a * (double)in_lo);
    if (!finite32(a) || !finite32(b))
        return fail(STRATA_EINVAL, "%s: [%s, %s] to [%s, %s] gives a scale of %s and an offset of %s; both must be finite",
                    op, fmt_v(in_lo, true).c_str(), fmt_v(in_hi, true).c_str(), fmt_v(out_lo, true).c_str(),
                    fmt_v(out_hi, true).c_str(), fmt_v(a, true).c_str(), fmt_v(b, true).c_str());
    return strata_stage_step(STRATA_VEC_AFFINE, -1, a, b, out);
}

// McCune and Keon's coefficients (terrain/heatload.go:104-108).
static const double kHeatLoadCoef[3][6] = {
    {-1.467, 1.582, -1.500, -0.262, 0.607, 0},
    {-1.236, 1.350, -1.376, -0.331, 0.375, 0},
    {0.339, 0.808, 0, -0.196, 0, -0.482},
};

extern "C" int strata_stage_heatload(strata_heatload_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    // heatLoadTerms (terrain/heatload.go:110-142), checked first as heatLoadOp does.
    if (o->equation < 0 || o->equation > 2)
        return fail(STRATA_EINVAL, "terrain: unknown HeatLoadEquation %d", o->equation);
    if (!(o->latitude >= -90 && o->latitude <= 90))
        return fail(STRATA_EINVAL, "terrain: Latitude must be in [-90, 90], got %s", fmt_v(o->latitude).c_str());
    const double* k = kHeatLoadCoef[o->equation];
    const double lat = std::fabs(o->latitude) * M_PI / 180;
    const double sin_l = std::sin(lat), cos_l = std::cos(lat);
    const double h = std::sqrt(2.0) / 2;
    double cos_c = h, sin_c = h;  // northeast
    const bool south = o->latitude < 0;
    if (o->radiation && !south) cos_c = 1, sin_c = 0;
    else if (o->radiation && south) cos_c = -1, sin_c = 0;
    else if (south) cos_c = -h, sin_c = h;
    const double kc = k[2] * sin_l + k[5];
    const double t[8] = {k[0], k[1] * cos_l, -kc * sin_c, kc * cos_c, k[3] * sin_l, k[4], cos_c, sin_c};
    memcpy(o->terms, t, sizeof t);
    int rc = fit_radius(o->fit_radius);
    if (rc) return rc;
    int base;
    if ((rc = deriv_stage(STRATA_OP_HEATLOAD, o->fit_radius, o->cell_size, o->cell_size_y, o->z_factor, out, &base)))
        return rc;
    out->kind = (o->linear && o->equation != 2) ? 1 : 0;
    out->table[0] = reinterpret_cast<const float*>(o->terms);
    out->table_len[0] = 16;
    return STRATA_OK;
}

extern "C" int strata_stage_orientation(const strata_orientation_options* o, strata_stage* out) {
    if (!o || !out) return fail(STRATA_EINVAL, "terrain: nil options");
    // orientationEast (terrain/orientation.go:45-53), checked first as orientationOp does.
    if (o->component != 0 && o->component != 1)
        return fail(STRATA_EINVAL, "terrain: unknown OrientationComponent %d", o->component);
    int rc = fit_radius(o->fit_radius);
    if (rc) return rc;
    int base;
    if ((rc = deriv_stage(STRATA_OP_ORIENTATION, o->fit_radius, o->cell_size, o->cell_size_y, o->z_factor, out,
                          &base)))
        return rc;
    out->kind = (o->component ? 1 : 0) | (o->unweighted ? 2 : 0);
    return STRATA_OK;
}

extern "C" int strata_focal_gaussian(int32_t radius, double sigma, float* taps) {
    int rc = check_focal_radius(radius);
    if (rc) return rc;
    if (!(sigma > 0) || std::isinf(sigma))
        return fail(STRATA_EINVAL, "focal: Gaussian sigma must be positive and finite, got %s", fmt_v(sigma).c_str());
    if (!taps) return fail(STRATA_EINVAL, "focal: nil taps");
    // focal.Gaussian (focal/separable.go:59-76).
    double g[2 * STRATA_MAX_RADIUS + 1];
    double sum = 0;
    for (int i = 0; i < 2 * radius + 1; i++) {
        double x = (double)(i - radius);
        g[i] = std::exp(-x * x / (2 * sigma * sigma));
        sum += g[i];
    }
    for (int i = 0; i < 2 * radius + 1; i++) taps[i] = (float)(g[i] / sum);
    return STRATA_OK;
}

// ---------------------------------------------------------------------------
// exec.ProcessChunked (internal/exec/chunked.go:33-464): tiles of the
// source, grown by the radius and clipped to the raster, are read into
// page-locked buffers, computed on the device, and handed to the sinks in
// plan order. Two buffer sets alternate, so tile i computes and copies
// while the host writes tile i-1 and reads tile i+1.

namespace {

int64_t round_up64(int64_t v) { return (v + 63) / 64 * 64; }

struct PinnedBuf {
    void* p = nullptr;
    size_t n = 0;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
    }
    int get(size_t bytes) {
        if (n >= bytes) return STRATA_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocDefault);
        if (e != cudaSuccess) return cuda_fail(e, "page-locked buffer");
        n = bytes;
        return STRATA_OK;
    }
};

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    int get(size_t bytes) {
        if (n >= bytes) return STRATA_OK;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 1);
        if (e != cudaSuccess) return cuda_fail(e, "device tile buffer");
        n = bytes;
        return STRATA_OK;
    }
};

// One tile's buffers: the input window and the outputs, host and device.
struct TileSet {
    PinnedBuf in_data, in_bits, out_data[2], out_bits[2];
    DevBuf d_in_data, d_in_bits, d_out_data[2], d_out_bits[2];
    cudaEvent_t done = nullptr;
    int64_t x0 = 0, y0 = 0, x1 = 0, y1 = 0;
    int64_t out_stride[2] = {0, 0};
    bool pending = false;
    ~TileSet() {
        if (done) cudaEventDestroy(done);
    }
};

// Where a chunked call's tiles come from and go to: the caller's callbacks
// (engine.RasterSource / RasterSink), or raw float32 files whose fill
// value becomes validity on the device (engine/raw.go).
struct ChunkIO {
    bool in_masked = false;  // the input tiles carry validity
    bool in_fill = false;    // ... derived on the device from in_fill_value
    float in_fill_value = 0;
    bool compact = false;  // tile rows at the tile's width (else masked rows start on 64-cell boundaries)
    // Fills the host tile buf (its cells, and its bits when the input is
    // masked and not derived) from the window at (x, y).
    std::function<int(const strata_raster& buf, int64_t x, int64_t y)> read;
    bool out_masked[2] = {false, false};  // output i's tiles carry validity
    bool out_fill[2] = {false, false};    // ... and take out_fill_value[i] under their invalid cells
    float out_fill_value[2] = {0, 0};
    // Takes output i's finished host tile (bits only for an output that is
    // masked and not filled).
    std::function<int(int i, const strata_raster& buf, int64_t x, int64_t y)> write;
    bool async_write = false;  // write a tile on a second thread while the next is read
};

// exec.ProcessChunked's tile loop (internal/exec/chunked.go:33-464) over
// two buffer sets: tile t reads with its halo, crosses to the device and
// computes while tile t - 1 goes to the sinks. p is planned for one input.
int run_chunked(strata_ctx* c, const LaunchParams& p, int nout, int64_t W, int64_t H, const ChunkIO& io,
                const strata_exec_opts* opts, strata_stats* stats) {
    const int ndst = nout;
    const int r = p.radius;
    const int64_t tw = (opts && opts->tile_width > 0) ? std::min<int64_t>(opts->tile_width, W) : W;
    const int64_t th = (opts && opts->tile_height > 0) ? std::min<int64_t>(opts->tile_height, H) : H;
    const int64_t tiles_x = (W + tw - 1) / tw;
    const int64_t ntiles = tiles_x * ((H + th - 1) / th);
    const int64_t inW = std::min(W, tw + 2 * r), inH = std::min(H, th + 2 * r);
    const bool in_masked = io.in_masked;
    const bool host_in_bits = in_masked && !io.in_fill;
    const int64_t in_stride = in_masked && !io.compact ? round_up64(inW) : inW;
    const int64_t in_cells = (inH - 1) * in_stride + inW;
    int rc;

    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard device_guard(c->device);
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;

    if (!c->chunk_sets)
        c->chunk_sets = std::shared_ptr<void>(new TileSet[2], [](void* q) { delete[] static_cast<TileSet*>(q); });
    TileSet* sets = static_cast<TileSet*>(c->chunk_sets.get());
    for (int k = 0; k < 2; k++) {
        TileSet& s = sets[k];
        s.pending = false;
        if ((rc = s.in_data.get((size_t)in_cells * 4)) || (rc = s.d_in_data.get((size_t)in_cells * 4))) return rc;
        if (in_masked) {
            size_t words = (size_t)((in_cells + 63) / 64);
            if ((rc = s.d_in_bits.get(words * 8))) return rc;
            if (host_in_bits && (rc = s.in_bits.get(words * 8))) return rc;
        }
        for (int i = 0; i < ndst; i++) {
            int64_t os = io.out_masked[i] && !io.compact ? round_up64(tw) : tw;
            int64_t oc = (th - 1) * os + tw;
            s.out_stride[i] = os;
            if ((rc = s.out_data[i].get((size_t)oc * 4)) || (rc = s.d_out_data[i].get((size_t)oc * 4))) return rc;
            if (io.out_masked[i]) {
                size_t words = (size_t)((oc + 63) / 64);
                if ((rc = s.d_out_bits[i].get(words * 8))) return rc;
                if (!io.out_fill[i] && (rc = s.out_bits[i].get(words * 8))) return rc;
            }
        }
        if (!s.done && cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) {
            s.done = nullptr;
            return fail(STRATA_ECUDA, "strata_cuda: cudaEventCreate");
        }
    }

    strata_stats local = {};
    int status = STRATA_OK;
    // Hands a finished tile to the sinks.
    auto write_tile = [&](TileSet& s) -> int {
        cudaError_t e = cudaEventSynchronize(s.done);
        if (e != cudaSuccess) return cuda_fail(e, "tile");
        for (int i = 0; i < ndst; i++) {
            strata_raster b = {};
            b.data = (float*)s.out_data[i].p;
            b.width = s.x1 - s.x0;
            b.height = s.y1 - s.y0;
            b.stride = s.out_stride[i];
            b.valid = io.out_masked[i] && !io.out_fill[i] ? (uint64_t*)s.out_bits[i].p : nullptr;
            const int wrc = io.write(i, b, s.x0, s.y0);
            if (wrc != STRATA_OK) return wrc;
        }
        int64_t cells = (s.x1 - s.x0) * (s.y1 - s.y0);
        local.sink_written += cells * 4 * ndst;
        local.cells += cells;
        local.ideal += cells * 4 * (1 + nout);
        local.kernel_written += cells * 4 * nout;
        local.tiles++;
        return STRATA_OK;
    };
    auto flush = [&](TileSet& s) -> int {
        if (!s.pending) return STRATA_OK;
        s.pending = false;
        return write_tile(s);
    };
    // With io.async_write a tile goes to the sinks on a second thread while
    // the next tile is read: its status, and its message (set on that
    // thread), come back when it is joined, before the set's output
    // buffers take another tile and before the call returns.
    std::future<std::pair<int, std::string>> writing;
    auto flush_async = [&](TileSet& s) {
        if (!s.pending) return;
        s.pending = false;
        TileSet* sp = &s;
        writing = std::async(std::launch::async, [&write_tile, sp]() {
            const int wrc = write_tile(*sp);
            return std::make_pair(wrc, wrc == STRATA_OK ? std::string() : g_err);
        });
    };
    auto join_write = [&]() -> int {
        if (!writing.valid()) return STRATA_OK;
        auto r = writing.get();
        if (r.first != STRATA_OK) g_err = r.second;
        return r.first;
    };

    const volatile int32_t* cancel = opts ? opts->cancel : nullptr;
    for (int64_t t = 0; t < ntiles && status == STRATA_OK; t++) {
        TileSet& s = sets[t & 1];
        // The set's previous tile (t - 2) must be with the sinks before its
        // buffers are reused; tile t - 1 is written while t computes. A
        // background write of tile t - 2 needs only its input copied in
        // before this read reuses the input buffers.
        if ((status = flush(s))) break;
        if (io.async_write) {
            const cudaError_t e = cudaEventSynchronize(s.done);
            if (e != cudaSuccess) {
                status = cuda_fail(e, "tile");
                break;
            }
        }
        if (cancel && *cancel) {
            status = STRATA_ECANCELED;
            break;
        }
        const int64_t x0 = (t % tiles_x) * tw, y0 = (t / tiles_x) * th;
        const int64_t x1 = std::min(x0 + tw, W), y1 = std::min(y0 + th, H);
        const int64_t rx0 = std::max<int64_t>(0, x0 - r), ry0 = std::max<int64_t>(0, y0 - r);
        const int64_t rx1 = std::min(W, x1 + r), ry1 = std::min(H, y1 + r);
        const int64_t ww = rx1 - rx0, wh = ry1 - ry0;
        const int64_t ws = in_masked && !io.compact ? round_up64(ww) : ww;
        const int64_t wcells = (wh - 1) * ws + ww;
        strata_raster b = {};
        b.data = (float*)s.in_data.p;
        b.width = ww;
        b.height = wh;
        b.stride = ws;
        b.valid = host_in_bits ? (uint64_t*)s.in_bits.p : nullptr;
        if (host_in_bits) memset(s.in_bits.p, 0, (size_t)((wcells + 63) / 64) * 8);
        if ((status = io.read(b, rx0, ry0)) != STRATA_OK) break;
        local.source_read += ww * wh * 4;
        cudaError_t e = cudaMemcpyAsync(s.d_in_data.p, s.in_data.p, (size_t)wcells * 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && host_in_bits)
            e = cudaMemcpyAsync(s.d_in_bits.p, s.in_bits.p, (size_t)((wcells + 63) / 64) * 8, cudaMemcpyHostToDevice,
                                st);
        if (e == cudaSuccess && in_masked && io.in_fill)
            strata::launch_fill_bits((const float*)s.d_in_data.p, wcells, io.in_fill_value, (uint32_t*)s.d_in_bits.p,
                                     st);
        for (int i = 0; i < ndst && e == cudaSuccess; i++)
            if (io.out_masked[i]) {
                int64_t oc = (y1 - y0 - 1) * s.out_stride[i] + (x1 - x0);
                e = cudaMemsetAsync(s.d_out_bits[i].p, 0, (size_t)((oc + 63) / 64) * 8, st);
            }
        if (e != cudaSuccess) {
            status = cuda_fail(e, "tile copy");
            break;
        }
        LaunchParams q = p;
        q.src = (const float*)s.d_in_data.p;
        q.src_stride = ws;
        q.src_x0 = rx0;
        q.src_y0 = ry0;
        q.src_w = ww;
        q.src_h = wh;
        q.dst0 = (float*)s.d_out_data[0].p;
        q.dst0_stride = s.out_stride[0];
        if (ndst > 1) {
            q.dst1 = (float*)s.d_out_data[1].p;
            q.dst1_stride = s.out_stride[1];
        }
        q.dst_x0 = x0;
        q.dst_y0 = y0;
        q.out_x0 = x0;
        q.out_y0 = y0;
        q.out_x1 = x1;
        q.out_y1 = y1;
        q.width = W;
        q.height = H;
        q.status = c->d_status;
        int64_t wc = 0;
        ValidityParams vp[2];
        const ValidityParams* vs[2] = {nullptr, nullptr};
        for (int i = 0; i < ndst; i++) {
            if (!io.out_masked[i]) continue;
            ValidityParams& v = vp[i];
            vs[i] = &v;
            memset(&v, 0, sizeof v);
            if (in_masked) {
                v.src_bits = (const uint32_t*)s.d_in_bits.p;
                v.src_off = 0;
                v.src_stride = ws;
                v.src_lo_word = 0;
                v.src_hi_word = (wcells - 1) >> 5;
            }
            v.src_x0 = rx0;
            v.src_y0 = ry0;
            v.dst_bits = (uint32_t*)s.d_out_bits[i].p;
            v.dst_off = 0;
            v.dst_stride = s.out_stride[i];
            v.dst_x0 = x0;
            v.dst_y0 = y0;
            v.out_x0 = x0;
            v.out_y0 = y0;
            v.out_x1 = x1;
            v.out_y1 = y1;
            v.width = W;
            v.height = H;
            v.radius = r;
            int64_t oc = (y1 - y0 - 1) * s.out_stride[i] + (x1 - x0);
            v.dst_lo_word = 0;
            v.dst_words = (oc + 31) >> 5;
        }
        int64_t nt = q.fit ? launch_fit(c, q, vs, st, &wc) : strata::launch_stage(q, vs, st, &wc);
        if (nt == -2) {
            status = fail(STRATA_ENOMEM, "engine: no device memory for the fit's sums");
            break;
        }
        if (nt < 0) {
            status = fail(STRATA_ENOTSUP, "engine: op %d at radius %d has no device kernel", p.op, p.radius);
            break;
        }
        local.bands += nt;
        local.kernel_read += wc * 4;
        for (int i = 0; i < ndst; i++)
            if (io.out_fill[i])
                strata::launch_fill_invalid((float*)s.d_out_data[i].p, s.out_stride[i], x1 - x0, y1 - y0,
                                            (const uint32_t*)s.d_out_bits[i].p, io.out_fill_value[i], st);
        // The set's output buffers still hold tile t - 2 while its
        // background write runs.
        if (io.async_write && (status = join_write())) break;
        for (int i = 0; i < ndst && e == cudaSuccess; i++) {
            int64_t oc = (y1 - y0 - 1) * s.out_stride[i] + (x1 - x0);
            e = cudaMemcpyAsync(s.out_data[i].p, s.d_out_data[i].p, (size_t)oc * 4, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess && io.out_masked[i] && !io.out_fill[i])
                e = cudaMemcpyAsync(s.out_bits[i].p, s.d_out_bits[i].p, (size_t)((oc + 63) / 64) * 8,
                                    cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(s.done, st);
        if (e != cudaSuccess) {
            status = cuda_fail(e, "tile");
            break;
        }
        s.x0 = x0;
        s.y0 = y0;
        s.x1 = x1;
        s.y1 = y1;
        s.pending = true;
        // Write the other set's tile (t - 1) while this one runs.
        if (io.async_write) flush_async(sets[(t + 1) & 1]);
        else if ((status = flush(sets[(t + 1) & 1]))) break;
    }
    // A tile still being written is the oldest.
    {
        const int wrc = join_write();
        if (status == STRATA_OK || status == STRATA_ECANCELED) status = wrc ? wrc : status;
    }
    // Tiles already computed are written in plan order, after a cancel too;
    // after a failure nothing more is written.
    if (status == STRATA_OK || status == STRATA_ECANCELED) {
        for (int64_t k = 0; k < 2; k++) {
            // the older pending tile first
            TileSet* a = &sets[0];
            TileSet* b2 = &sets[1];
            TileSet* first = (a->pending && b2->pending) ? ((a->y0 < b2->y0 || (a->y0 == b2->y0 && a->x0 < b2->x0)) ? a : b2)
                                                          : (a->pending ? a : b2);
            int frc = flush(*first);
            if (frc) {
                status = frc;
                break;
            }
        }
    } else {
        cudaStreamSynchronize(st);
    }
    if (stats) {
        stats->cells += local.cells;
        stats->ideal += local.ideal;
        stats->tiles += local.tiles;
        stats->bands += local.bands;
        stats->source_read += local.source_read;
        stats->sink_written += local.sink_written;
        stats->kernel_read += local.kernel_read;
        stats->kernel_written += local.kernel_written;
    }
    if (status == STRATA_OK) status = take_status(c, st);
    if (status == STRATA_ECANCELED) return fail(STRATA_ECANCELED, "context canceled");
    return status;
}

// Reads or writes n bytes at off of fd, retrying short transfers; returns
// the bytes moved (less than n at the end of the file or on an error, with
// errno set for an error).
int64_t raw_io(bool write, int fd, char* p, int64_t n, int64_t off) {
    int64_t done = 0;
    while (done < n) {
        const size_t k = (size_t)std::min<int64_t>(n - done, (int64_t)1 << 30);
        const ssize_t got = write ? pwrite(fd, p + done, k, (off_t)(off + done)) : pread(fd, p + done, k, (off_t)(off + done));
        if (got < 0 && errno == EINTR) continue;
        if (got <= 0) {
            if (got == 0) errno = 0;
            break;
        }
        done += got;
    }
    return done;
}

// raw_io over large spans in parts of at least 2 MiB on up to 8 threads
// (a page-cache copy runs at one core's memory bandwidth). Returns whether
// every byte moved, with the first failing part's errno in *err.
bool raw_io_parallel(bool write, int fd, char* p, int64_t n, int64_t off, int* err) {
    constexpr int64_t kPart = (int64_t)2 << 20;
    const int parts = (int)std::min<int64_t>(8, std::max<int64_t>(1, n / kPart));
    *err = 0;
    if (parts == 1) {
        const bool ok = raw_io(write, fd, p, n, off) == n;
        if (!ok) *err = errno;
        return ok;
    }
    const int64_t step = (n / parts + 4095) / 4096 * 4096;
    std::vector<std::thread> threads;
    std::vector<int> errs((size_t)parts, 0);
    std::vector<char> oks((size_t)parts, 1);
    for (int k = 0; k < parts; k++) {
        const int64_t a = k * step, b = std::min(n, a + step);
        if (a >= b) break;
        threads.emplace_back([=, &errs, &oks]() {
            if (raw_io(write, fd, p + a, b - a, off + a) != b - a) {
                oks[(size_t)k] = 0;
                errs[(size_t)k] = errno;
            }
        });
    }
    for (auto& t : threads) t.join();
    for (int k = 0; k < parts; k++)
        if (!oks[(size_t)k]) {
            *err = errs[(size_t)k];
            return false;
        }
    return true;
}

std::string rows_name(int64_t y, int64_t k) {
    char b[64];
    if (k == 1) snprintf(b, sizeof b, "row %lld", (long long)y);
    else snprintf(b, sizeof b, "rows %lld to %lld", (long long)y, (long long)(y + k - 1));
    return b;
}

// The rows of tile buf at (x, y) of a raw file: one call for rows that are
// consecutive both in the file and in buf (a window as wide as the file
// into a buffer without row padding), else a call per row
// (engine/raw.go:74-111, 195-239).
int raw_rows(bool write, const strata_raw_file& f, const strata_raster& buf, int64_t x, int64_t y) {
    const bool whole = buf.width == f.width && buf.stride == buf.width;
    const int64_t per = whole ? buf.height : 1;
    for (int64_t row = 0; row < buf.height; row += per) {
        const int64_t k = std::min(per, buf.height - row);
        const int64_t n = ((k - 1) * buf.stride + buf.width) * 4;
        const int64_t off = f.offset + 4 * ((y + row) * f.width + x);
        int err = 0;
        if (!raw_io_parallel(write, f.fd, (char*)(buf.data + row * buf.stride), n, off, &err)) {
            if (write)
                return fail(STRATA_EIO, "engine: raw sink: writing %s: %s", rows_name(y + row, k).c_str(),
                            err ? strerror(err) : "short write");
            return fail(STRATA_EIO, "engine: raw source: reading %s: %s", rows_name(y + row, k).c_str(),
                        err ? strerror(err) : "unexpected EOF");
        }
    }
    return STRATA_OK;
}

// NewRawSource / NewRawSink's checks (engine/raw.go:278-289).
int check_raw(const char* fn, const strata_raw_file& f) {
    if (f.fd < 0) return fail(STRATA_EINVAL, "engine: %s: nil file", fn);
    if (f.width <= 0 || f.height <= 0)
        return fail(STRATA_EINVAL, "engine: %s: dimensions must be positive, got %lld×%lld", fn, (long long)f.width,
                    (long long)f.height);
    if ((uint64_t)f.width > (uint64_t)INT64_MAX / 4 / (uint64_t)f.height)
        return fail(STRATA_EINVAL, "engine: %s: %lld×%lld cells do not fit in a file", fn, (long long)f.width,
                    (long long)f.height);
    if (f.offset < 0) return fail(STRATA_EINVAL, "engine: %s: negative offset %lld", fn, (long long)f.offset);
    return STRATA_OK;
}

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "raw files are read in place: a little-endian host");

}  // namespace

extern "C" int strata_process_chunked(strata_ctx* c, const strata_stage* stages, int nstages,
                                      const strata_source* src, int nsrc, const strata_sink* dst, int ndst,
                                      const strata_exec_opts* opts, strata_stats* stats) {
    if (!c) return fail(STRATA_EINVAL, "engine: nil context");
    LaunchParams p;
    int nout = 0;
    int rc = plan_stages(stages, nstages, p, &nout);
    if (rc) return rc;
    if (p.ninputs > 1 || nsrc > 1)
        return fail(STRATA_ENOTSUP, "engine: a chain over several inputs has no chunked form on the gpu backend");
    if ((rc = check_opts(opts))) return rc;
    if (nsrc != 1 || ndst != nout || !src || !dst)
        return fail(STRATA_EINVAL, "engine: kernel takes 1 inputs and %d outputs, got %d and %d", nout, nsrc, ndst);
    for (int i = 0; i < ndst; i++)
        if (!dst[i].write) return fail(STRATA_EINVAL, "engine: dst[%d] is a nil sink", i);
    if (!src[0].read) return fail(STRATA_EINVAL, "engine: src[0] is a nil source");
    const int64_t W = dst[0].width, H = dst[0].height;
    if (W <= 0 || H <= 0)
        return fail(STRATA_EINVAL, "engine: dst[0] is %lld×%lld; sizes must be positive", (long long)W, (long long)H);
    if (src[0].width != W || src[0].height != H)
        return fail(STRATA_EINVAL, "engine: src[0] is %lld×%lld, dst[0] is %lld×%lld", (long long)src[0].width,
                    (long long)src[0].height, (long long)W, (long long)H);
    for (int i = 0; i < ndst; i++) {
        if (dst[i].width != W || dst[i].height != H)
            return fail(STRATA_EINVAL, "engine: dst[%d] is %lld×%lld, dst[0] is %lld×%lld", i, (long long)dst[i].width,
                        (long long)dst[i].height, (long long)W, (long long)H);
        if (src[0].masked && !dst[i].masked)
            return fail(STRATA_EINVAL, "engine: a source is Masked but dst[%d] is not; its validity would be lost", i);
    }
    ChunkIO io;
    io.in_masked = src[0].masked != 0;
    io.read = [&](const strata_raster& b, int64_t x, int64_t y) -> int {
        if (src[0].read(src[0].user, &b, x, y) != 0)
            return fail(STRATA_EIO, "engine: reading src[0] at (%lld, %lld) failed", (long long)x, (long long)y);
        return STRATA_OK;
    };
    for (int i = 0; i < ndst; i++) io.out_masked[i] = dst[i].masked != 0;
    io.write = [&](int i, const strata_raster& b, int64_t x, int64_t y) -> int {
        if (dst[i].write(dst[i].user, &b, x, y) != 0)
            return fail(STRATA_EIO, "engine: writing dst[%d] at (%lld, %lld) failed", i, (long long)x, (long long)y);
        return STRATA_OK;
    };
    return run_chunked(c, p, nout, W, H, io, opts, stats);
}

extern "C" int strata_process_raw(strata_ctx* c, const strata_stage* stages, int nstages, const strata_raw_file* src,
                                  int nsrc, const strata_raw_file* dst, int ndst, const strata_exec_opts* opts,
                                  strata_stats* stats) {
    if (!c) return fail(STRATA_EINVAL, "engine: nil context");
    LaunchParams p;
    int nout = 0;
    int rc = plan_stages(stages, nstages, p, &nout);
    if (rc) return rc;
    if (p.ninputs > 1 || nsrc > 1)
        return fail(STRATA_ENOTSUP, "engine: a chain over several inputs has no chunked form on the gpu backend");
    if ((rc = check_opts(opts))) return rc;
    if (nsrc != 1 || ndst != nout || !src || !dst)
        return fail(STRATA_EINVAL, "engine: kernel takes 1 inputs and %d outputs, got %d and %d", nout, nsrc, ndst);
    if ((rc = check_raw("NewRawSource", src[0]))) return rc;
    const int64_t W = src[0].width, H = src[0].height;
    for (int i = 0; i < ndst; i++) {
        if ((rc = check_raw("NewRawSink", dst[i]))) return rc;
        if (dst[i].width != W || dst[i].height != H)
            return fail(STRATA_EINVAL, "engine: dst[%d] is %lld×%lld, src[0] is %lld×%lld", i, (long long)dst[i].width,
                        (long long)dst[i].height, (long long)W, (long long)H);
        if (src[0].has_fill && !dst[i].has_fill)
            return fail(STRATA_EINVAL, "engine: a source is Masked but dst[%d] is not; its validity would be lost", i);
    }
    ChunkIO io;
    io.compact = true;
    io.in_masked = io.in_fill = src[0].has_fill != 0;
    io.in_fill_value = src[0].fill;
    io.read = [&](const strata_raster& b, int64_t x, int64_t y) { return raw_rows(false, src[0], b, x, y); };
    for (int i = 0; i < ndst; i++) {
        io.out_masked[i] = io.out_fill[i] = dst[i].has_fill != 0;
        io.out_fill_value[i] = dst[i].fill;
    }
    io.write = [&](int i, const strata_raster& b, int64_t x, int64_t y) { return raw_rows(true, dst[i], b, x, y); };
    io.async_write = true;
    return run_chunked(c, p, nout, W, H, io, opts, stats);
}

// ---------------------------------------------------------------------------
// terrain.Features / terrain.Surface (terrain/features.go:60-92,
// terrain/surface.go:57-98): several pipelines over one input in one
// call. A host input crosses to the device once; each output's copy back
// runs on a second stream while the next pipeline computes.

extern "C" int strata_process_features(strata_ctx* c, const strata_stage* stages, const int32_t* counts,
                                       int nfeatures, const strata_raster* src, const strata_raster* dst,
                                       int ndst, const strata_exec_opts* opts, strata_stats* stats) {
    if (!c) return fail(STRATA_EINVAL, "engine: nil context");
    if (nfeatures < 1 || !stages || !counts || !src || !dst)
        return fail(STRATA_EINVAL, "terrain: Features has no outputs");
    int rc;
    if ((rc = check_opts(opts))) return rc;
    // Resolve every feature's pipeline and its outputs.
    std::vector<LaunchParams> plans((size_t)nfeatures);
    std::vector<int> nouts((size_t)nfeatures), first((size_t)nfeatures);
    int off = 0, outs = 0, rmax = 0;
    for (int f = 0; f < nfeatures; f++) {
        if (counts[f] < 1) return fail(STRATA_EINVAL, "terrain: Features output %d has no Op", f);
        if ((rc = plan_stages(stages + off, counts[f], plans[(size_t)f], &nouts[(size_t)f]))) return rc;
        if (plans[(size_t)f].ninputs > 1)
            return fail(STRATA_EINVAL, "engine: a feature reads one input, feature %d's chain reads %d", f,
                        plans[(size_t)f].ninputs);
        first[(size_t)f] = outs;
        outs += nouts[(size_t)f];
        off += counts[f];
        rmax = std::max(rmax, plans[(size_t)f].radius);
    }
    if (ndst != outs)
        return fail(STRATA_EINVAL, "engine: the features write %d outputs, got %d rasters", outs, ndst);
    // The checks of one ProcessN call with every output (the pipeline's
    // radius is the largest of its stages').
    if ((rc = check_operands(src, 1, dst, ndst, ndst, rmax))) return rc;

    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard device_guard(c->device);
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    cudaStream_t cs = c->copy_stream;
    const int64_t W = src[0].width, H = src[0].height;
    DevOperand ds;
    if ((rc = stage_in(c, st, src[0], 0, true, &ds))) return rc;
    std::vector<DevOperand> dd((size_t)ndst);
    for (int i = 0; i < ndst; i++)
        if ((rc = stage_in(c, st, dst[i], 2 + 2 * i, false, &dd[(size_t)i]))) return rc;
    if ((rc = ensure_edges(c, (size_t)ndst))) return rc;
    std::vector<cudaEvent_t> events;
    auto cleanup = [&] {
        for (auto e : events) cudaEventDestroy(e);
    };
    int64_t bands = 0, window = 0;
    // Starts the copies back of outputs [o, o + n) once the work queued on st
    // so far is done, on the copy stream, so they overlap the next kernels.
    auto copy_back = [&](int o, int n, cudaStream_t from) -> int {
        bool any_host = false;
        for (int i = o; i < o + n; i++) any_host = any_host || !dst[i].on_device;
        if (!any_host) return STRATA_OK;
        cudaEvent_t ev;
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "event");
        events.push_back(ev);
        cudaEventRecord(ev, from);
        cudaStreamWaitEvent(cs, ev, 0);
        for (int i = o; i < o + n; i++) {
            if (dst[i].on_device) continue;
            const DevOperand& d = dd[(size_t)i];
            e = data_back(dst[i], d, cs);
            if (e == cudaSuccess && dst[i].valid) e = mask_back(dst[i], d, c->h_edges + 2 * i, cs);
            if (e != cudaSuccess) return cuda_fail(e, "copy to host");
        }
        return STRATA_OK;
    };
    for (int f = 0; f < nfeatures; f++) {
        LaunchParams& p = plans[(size_t)f];
        const int o = first[(size_t)f];
        p.src = ds.data;
        p.src_stride = ds.stride;
        p.src_x0 = p.src_y0 = 0;
        p.src_w = W;
        p.src_h = H;
        p.dst0 = dd[(size_t)o].data;
        p.dst0_stride = dd[(size_t)o].stride;
        if (nouts[(size_t)f] > 1) {
            p.dst1 = dd[(size_t)o + 1].data;
            p.dst1_stride = dd[(size_t)o + 1].stride;
        }
        p.dst_x0 = p.dst_y0 = 0;
        p.width = W;
        p.height = H;
        p.out_x0 = 0;
        p.out_x1 = W;
        p.out_y0 = 0;
        p.out_y1 = H;
        p.status = c->d_status;
    }
    // The memory-bound radius-1 features whose rows the TMA march takes run
    // as one fused pass (one read of the source, Horn's differences formed
    // once; features.cu says which); the others, and all of them when fewer
    // than two fuse, run one by one.
    std::vector<char> done((size_t)nfeatures, 0);
    {
        std::unique_ptr<strata::FeaturesParams> fp(new strata::FeaturesParams);
        memset(fp.get(), 0, sizeof(strata::FeaturesParams));
        std::vector<int> group;
        for (int f = 0; f < nfeatures; f++) {
            const LaunchParams& p = plans[(size_t)f];
            const int q = strata::feature_slot(p);
            if (q < 0 || fp->f[q].on) continue;
            strata::FeatureSlot& F = fp->f[q];
            F.on = 1;
            memcpy(F.k, p.k, sizeof F.k);
            if (p.nepi == 1) {
                F.nb = p.epi[0].n;
                memcpy(F.t, p.epi[0].a, sizeof(float) * (size_t)F.nb);
                memcpy(F.v, p.epi[0].b, sizeof(float) * (size_t)(F.nb + 1));
            }
            if (q == strata::kFGradient || q == strata::kFSlopeClass || q == strata::kFSlopePercent) fp->horn = 1;
            else fp->window = 1;
            for (int k = 0; k < nouts[(size_t)f]; k++) {
                const int i = first[(size_t)f] + k;
                F.data[k] = dd[(size_t)i].data;
                F.stride[k] = dd[(size_t)i].stride;
                if (dst[i].valid) {
                    F.bits[k] = dd[(size_t)i].bits;
                    F.bit_off[k] = dd[(size_t)i].bit_off;
                    F.bit_stride[k] = dd[(size_t)i].stride;
                    fp->masked = 1;
                }
            }
            group.push_back(f);
        }
        if (group.size() >= 2) {
            fp->g = plans[(size_t)group[0]];
            LaunchParams& g = fp->g;
            memset(&g.vf, 0, sizeof g.vf);
            if (src[0].valid) {
                g.vf.src_bits = ds.bits;
                g.vf.src_off = ds.bit_off;
                g.vf.src_stride = ds.stride;
                g.vf.src_lo_word = ds.lo_word;
                g.vf.src_hi_word = ds.hi_word;
            }
            int64_t wc = 0;
            const int64_t t = strata::launch_features(*fp, st, &wc);
            if (t >= 0) {
                bands += t;
                window += wc;
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) {
                    cleanup();
                    return cuda_fail(e, "kernel launch");
                }
                for (int f : group) {
                    done[(size_t)f] = 1;
                    if ((rc = copy_back(first[(size_t)f], nouts[(size_t)f], st))) {
                        cleanup();
                        return rc;
                    }
                }
            }
        }
    }
    // The features that run as their own launches alternate between the
    // call's stream and a second one, so that one kernel's last wave
    // overlaps the next kernel's first; Wood's fit keeps to the call's
    // stream (its sums share the context's scratch).
    int own = 0;
    for (int f = 0; f < nfeatures; f++) own += !done[(size_t)f] && !plans[(size_t)f].fit;
    cudaStream_t lanes[2] = {st, st};
    if (own >= 2) {
        if (!c->aux_stream && (cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking) != cudaSuccess ||
                               cudaEventCreateWithFlags(&c->aux_fork, cudaEventDisableTiming) != cudaSuccess ||
                               cudaEventCreateWithFlags(&c->aux_join, cudaEventDisableTiming) != cudaSuccess)) {
            cudaGetLastError();
            if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
            if (c->aux_fork) cudaEventDestroy(c->aux_fork);
            c->aux_stream = nullptr;
            c->aux_fork = nullptr;
        }
        if (c->aux_stream && c->aux_join) {
            lanes[1] = c->aux_stream;
            cudaEventRecord(c->aux_fork, st);
            cudaStreamWaitEvent(c->aux_stream, c->aux_fork, 0);
        }
    }
    int lane = 0;
    for (int f = 0; f < nfeatures; f++) {
        if (done[(size_t)f]) continue;
        LaunchParams& p = plans[(size_t)f];
        const int o = first[(size_t)f];
        const cudaStream_t fs = p.fit ? st : lanes[lane];
        if (!p.fit) lane ^= 1;
        int64_t wc = 0;
        ValidityParams vp[2];
        const ValidityParams* vs[2] = {nullptr, nullptr};
        for (int i = o; i < o + nouts[(size_t)f]; i++) {
            if (!dst[i].valid) continue;
            fill_validity(vp[i - o], ds, src[0].valid != nullptr, dd[(size_t)i], span_cells(dst[i]), W, H, p.radius,
                          0, H);
            vs[i - o] = &vp[i - o];
        }
        int64_t t = p.fit ? launch_fit(c, p, vs, st, &wc) : strata::launch_stage(p, vs, fs, &wc);
        if (t < 0) {
            if (lanes[1] != st) {
                cudaEventRecord(c->aux_join, lanes[1]);
                cudaStreamWaitEvent(st, c->aux_join, 0);
            }
            cleanup();
            if (t == -2) return fail(STRATA_ENOMEM, "engine: no device memory for the fit's sums");
            return fail(STRATA_ENOTSUP, "engine: op %d at radius %d has no device kernel", p.op, p.radius);
        }
        bands += t;
        window += wc;
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            cleanup();
            return cuda_fail(e, "kernel launch");
        }
        // The outputs' copies back overlap the next feature's kernels.
        if ((rc = copy_back(o, nouts[(size_t)f], fs))) {
            cleanup();
            return rc;
        }
    }
    if (lanes[1] != st) {
        cudaEventRecord(c->aux_join, lanes[1]);
        cudaStreamWaitEvent(st, c->aux_join, 0);
    }
    cudaError_t e = cudaStreamSynchronize(cs);
    cleanup();
    if (e != cudaSuccess) return cuda_fail(e, "copy to host");
    bool all_device = src[0].on_device != 0;
    for (int i = 0; i < ndst; i++) all_device = all_device && dst[i].on_device;
    if (!(all_device && opts && (opts->flags & STRATA_EXEC_ASYNC)))
        if ((rc = take_status(c, st))) return rc;
    for (int i = 0; i < ndst; i++)
        if (!dst[i].on_device && dst[i].valid) merge_edges(dst[i], dd[(size_t)i], c->h_edges + 2 * i);
    if (stats) {
        const int64_t cells = W * H;
        stats->cells += cells;
        stats->ideal += cells * 4 * (1 + ndst);
        stats->bands += bands;
        stats->kernel_read += window * 4;
        stats->kernel_written += cells * 4 * ndst;
    }
    return STRATA_OK;
}

// ---------------------------------------------------------------------------
// Batches: many device-resident rasters of mixed sizes and ops, planned
// once (descriptors uploaded, one persistent kernel per op class captured
// in a CUDA graph) and run with one graph launch.

namespace {

bool aligned16_host(const void* q) { return ((uintptr_t)q & 15) == 0; }

// Checks batch item i as strata_process would and resolves it into a
// planned-to-be descriptor (its requested band in b.th). Allocates nothing.
int fill_batch_item(strata_ctx* c, const strata_batch_item& it, int i, strata::BatchItem& b, int* nout_out) {
    LaunchParams p;
    int nout = 0, rc;
    if ((rc = plan_stages(it.stages, it.nstages, p, &nout))) return rc;
    if ((rc = check_operands(&it.src, 1, it.dst, nout, nout, p.radius, p.ninputs))) return rc;
    if (!it.src.on_device || !it.dst[0].on_device || (nout > 1 && !it.dst[1].on_device))
        return fail(STRATA_EINVAL, "engine: batch raster %d: the rasters of a batch must be on the device", i);
    if (is_pointwise((uint32_t)p.op))
        return fail(STRATA_ENOTSUP, "engine: batch raster %d: a pointwise op alone has no batch kernel", i);
    if (p.fit)
        return fail(STRATA_ENOTSUP, "engine: batch raster %d: Wood's fit (FitRadius > 0) has no batch kernel", i);
    if (it.tile_height < 0 || it.tile_height > 1024)
        return fail(STRATA_EINVAL, "engine: batch raster %d: band of %d rows (0 to 1024)", i, it.tile_height);
    DevOperand ds, dd[2];
    if ((rc = stage_in(c, nullptr, it.src, 0, false, &ds))) return rc;
    for (int k = 0; k < nout; k++)
        if ((rc = stage_in(c, nullptr, it.dst[k], 0, false, &dd[k]))) return rc;
    const int64_t W = it.src.width, H = it.src.height;
    p.src = ds.data;
    p.src_stride = ds.stride;
    p.src_x0 = p.src_y0 = 0;
    p.src_w = W;
    p.src_h = H;
    p.dst0 = dd[0].data;
    p.dst0_stride = dd[0].stride;
    if (nout > 1) {
        p.dst1 = dd[1].data;
        p.dst1_stride = dd[1].stride;
    }
    p.dst_x0 = p.dst_y0 = 0;
    p.width = W;
    p.height = H;
    p.out_x0 = p.out_y0 = 0;
    p.out_x1 = W;
    p.out_y1 = H;
    memset(&b, 0, sizeof b);
    b.p = p;
    for (int k = 0; k < nout; k++) {
        if (!it.dst[k].valid) continue;
        fill_validity(b.v[b.nvalid], ds, it.src.valid != nullptr, dd[k], span_cells(it.dst[k]), W, H, p.radius, 0, H);
        b.nvalid++;
    }
    b.th = it.tile_height;
    b.vec = aligned16_host(p.src) && aligned16_host(p.dst0) && !(p.src_stride & 3) && !(p.dst0_stride & 3) &&
            (nout < 2 || (aligned16_host(p.dst1) && !(p.dst1_stride & 3)));
    *nout_out = nout;
    return STRATA_OK;
}

// Launches planned classes on stream st, each data class and the validity
// on branches of their own (forked from and joined back to st, so a
// capture of st records them as parallel graph nodes).
int launch_planned(const strata::BatchClass* cls, int nc, const strata::BatchItem* d_items,
                   const strata::ValidityClass* vcls, int nvc, const strata::ValidityItem* d_vitems, cudaStream_t st,
                   cudaStream_t* branch, int nbranch, cudaEvent_t* ev) {
    cudaError_t e = cudaEventRecord(ev[0], st);
    for (int k = 0; k < nbranch && e == cudaSuccess; k++) e = cudaStreamWaitEvent(branch[k], ev[0], 0);
    if (e != cudaSuccess) return cuda_fail(e, "batch fork");
    for (int i = 0; i < nc; i++)
        if (!strata::launch_batch_class(cls[i], d_items, branch[i % nbranch]))
            return fail(STRATA_ENOTSUP, "engine: an op of the batch has no batch kernel");
    for (int i = 0; i < nvc; i++) strata::launch_batch_validity(vcls[i], d_vitems, branch[(nc + i) % nbranch]);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "batch launch");
    for (int k = 0; k < nbranch && e == cudaSuccess; k++) {
        e = cudaEventRecord(ev[1 + k], branch[k]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev[1 + k], 0);
    }
    if (e != cudaSuccess) return cuda_fail(e, "batch join");
    return STRATA_OK;
}

constexpr int kBranches = 4;

}  // namespace

struct strata_batch {
    strata_ctx* ctx = nullptr;
    strata::BatchItem* d_items = nullptr;       // the descriptors, on the device
    strata::ValidityItem* d_vitems = nullptr;  // the validity descriptors
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int classes = 0;
    int64_t tiles = 0, cells = 0, window = 0;
    int64_t out_cells = 0, in_bytes = 0, out_bytes = 0;
};

extern "C" int strata_batch_create(strata_ctx* c, const strata_batch_item* items, int nitems, strata_batch** out) {
    if (!c || !out) return fail(STRATA_EINVAL, "engine: nil context");
    *out = nullptr;
    if (nitems < 1 || !items) return fail(STRATA_EINVAL, "engine: a batch needs at least one raster");
    std::lock_guard<std::mutex> lock(c->mu);
    DeviceGuard device_guard(c->device);
    std::vector<strata::BatchItem> host((size_t)nitems);
    int64_t cells = 0, in_bytes = 0, out_bytes = 0;
    for (int i = 0; i < nitems; i++) {
        int nout = 0, rc;
        if ((rc = fill_batch_item(c, items[i], i, host[(size_t)i], &nout))) return rc;
        host[(size_t)i].p.status = c->d_status;
        const int64_t n = items[i].src.width * items[i].src.height;
        cells += n;
        in_bytes += n * 4;
        out_bytes += n * 4 * nout;
    }
    std::vector<int> order((size_t)nitems);
    std::vector<strata::BatchClass> cls((size_t)nitems);
    int64_t window = 0;
    const int nc = strata::batch_plan(host.data(), nitems, order.data(), cls.data(), &window);
    if (nc < 0) return fail(STRATA_ENOTSUP, "engine: an op of the batch has no batch kernel");
    std::vector<strata::ValidityItem> vitems((size_t)(2 * nitems));
    strata::ValidityClass vcls[STRATA_MAX_RADIUS + 1];
    int nvc = 0;
    const int nv = strata::batch_plan_validity(host.data(), nitems, vitems.data(), vcls, &nvc);

    auto* B = new strata_batch;
    B->ctx = c;
    B->classes = nc;
    B->cells = cells;
    B->in_bytes = in_bytes;
    B->out_bytes = out_bytes;
    B->window = window;
    for (int i = 0; i < nc; i++) B->tiles += cls[(size_t)i].total;
    cudaError_t e = cudaMalloc(&B->d_items, sizeof(strata::BatchItem) * (size_t)nitems);
    if (e == cudaSuccess)
        e = cudaMemcpy(B->d_items, host.data(), sizeof(strata::BatchItem) * (size_t)nitems, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nv > 0) e = cudaMalloc(&B->d_vitems, sizeof(strata::ValidityItem) * (size_t)nv);
    if (e == cudaSuccess && nv > 0)
        e = cudaMemcpy(B->d_vitems, vitems.data(), sizeof(strata::ValidityItem) * (size_t)nv, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        strata_batch_destroy(B);
        return cuda_fail(e, "batch descriptors");
    }
    // Capture every class's persistent kernel into one graph, the classes
    // on parallel branches.
    cudaStream_t cap = nullptr, br[kBranches] = {};
    cudaEvent_t ev[1 + kBranches] = {};
    e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    for (int k = 0; k < kBranches && e == cudaSuccess; k++) e = cudaStreamCreateWithFlags(&br[k], cudaStreamNonBlocking);
    for (int k = 0; k < 1 + kBranches && e == cudaSuccess; k++) e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
    int rc = STRATA_OK;
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = launch_planned(cls.data(), nc, B->d_items, vcls, nvc, B->d_vitems, cap, br, kBranches, ev);
        cudaError_t e2 = cudaStreamEndCapture(cap, &B->graph);
        if (rc == STRATA_OK && e2 == cudaSuccess) e2 = cudaGraphInstantiate(&B->exec, B->graph, 0);
        if (rc == STRATA_OK && e2 != cudaSuccess) rc = cuda_fail(e2, "batch graph");
    } else {
        rc = cuda_fail(e, "batch capture");
    }
    for (int k = 0; k < 1 + kBranches; k++)
        if (ev[k]) cudaEventDestroy(ev[k]);
    for (int k = 0; k < kBranches; k++)
        if (br[k]) cudaStreamDestroy(br[k]);
    if (cap) cudaStreamDestroy(cap);
    if (rc != STRATA_OK) {
        cudaGetLastError();
        strata_batch_destroy(B);
        return rc;
    }
    *out = B;
    return STRATA_OK;
}

extern "C" int strata_batch_run(strata_batch* B, void* stream, int synchronize) {
    if (!B) return fail(STRATA_EINVAL, "engine: nil batch");
    DeviceGuard device_guard(B->ctx->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : B->ctx->stream;
    cudaError_t e = cudaGraphLaunch(B->exec, st);
    if (e != cudaSuccess) return cuda_fail(e, "batch launch");
    if (synchronize) return take_status(B->ctx, st);
    return STRATA_OK;
}

extern "C" int strata_batch_info(const strata_batch* B, strata_stats* stats, int* classes) {
    if (!B) return fail(STRATA_EINVAL, "engine: nil batch");
    if (classes) *classes = B->classes;
    if (stats) {
        stats->cells += B->cells;
        stats->ideal += B->in_bytes + B->out_bytes;
        stats->bands += B->tiles;
        stats->kernel_read += B->window * 4;
        stats->kernel_written += B->out_bytes;
    }
    return STRATA_OK;
}

extern "C" void strata_batch_destroy(strata_batch* B) {
    if (!B) return;
    DeviceGuard device_guard(B->ctx->device);
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    if (B->d_items) cudaFree(B->d_items);
    if (B->d_vitems) cudaFree(B->d_vitems);
    delete B;
}

// ---------------------------------------------------------------------------
// A batch run without allocation: the descriptors go to a fixed scratch
// area in the module's static device memory instead of cudaMalloc'd
// tables, and the class kernels launch straight onto the caller's stream
// (no graph). The scratch is one per device: calls on one stream are
// ordered by it, calls on different streams that overlap on the device
// race on it.

namespace {

constexpr size_t kScratchHead = 256;  // the status word, padded so the tables stay 256-byte aligned
constexpr size_t kItemBytes = sizeof(strata::BatchItem) * STRATA_NOALLOC_BATCH_MAX;
constexpr size_t kScratchBytes = kScratchHead + kItemBytes + sizeof(strata::ValidityItem) * 2 * STRATA_NOALLOC_BATCH_MAX;
static_assert(kItemBytes % 16 == 0, "the validity table starts on a 16-byte boundary");
static __device__ __align__(256) unsigned char g_batch_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
struct ScratchSlot {
    std::once_flag once;
    cudaError_t err = cudaSuccess;
    unsigned char* ptr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];

// Host staging of the descriptors and the plan; one call at a time.
std::mutex g_noalloc_mu;
strata::BatchItem g_noalloc_items[STRATA_NOALLOC_BATCH_MAX];
strata::ValidityItem g_noalloc_vitems[2 * STRATA_NOALLOC_BATCH_MAX];
int g_noalloc_order[STRATA_NOALLOC_BATCH_MAX];
strata::BatchClass g_noalloc_classes[STRATA_NOALLOC_BATCH_MAX];

// The device address of the scratch area, looked up once per device with
// that device current (the caller's guard makes it current), and its
// status word cleared.
int scratch_address(int device, unsigned char** ptr) {
    if (device < 0 || device >= kMaxDevices) return fail(STRATA_EINVAL, "engine: device %d out of range", device);
    ScratchSlot& s = g_scratch[device];
    std::call_once(s.once, [&] {
        s.err = cudaGetSymbolAddress((void**)&s.ptr, g_batch_scratch);
        if (s.err == cudaSuccess) s.err = cudaMemset(s.ptr, 0, sizeof(int));
    });
    if (s.err != cudaSuccess) return cuda_fail(s.err, "batch scratch address");
    *ptr = s.ptr;
    return STRATA_OK;
}

}  // namespace

extern "C" int strata_batch_run_noalloc(strata_ctx* c, const strata_batch_item* items, int nitems, void* stream,
                                        int synchronize) {
    if (!c) return fail(STRATA_EINVAL, "engine: nil context");
    if (nitems < 1 || !items) return fail(STRATA_EINVAL, "engine: a batch needs at least one raster");
    if (nitems > STRATA_NOALLOC_BATCH_MAX)
        return fail(STRATA_EINVAL, "engine: %d rasters exceed the %d a batch without allocation can hold", nitems,
                    STRATA_NOALLOC_BATCH_MAX);
    std::lock_guard<std::mutex> lock(c->mu);
    std::lock_guard<std::mutex> staging(g_noalloc_mu);
    DeviceGuard device_guard(c->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    // The descriptors go up from the library's pageable host staging,
    // which the next call rewrites: a capture would record those copies by
    // host address and replay whatever the latest call left there.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) return cuda_fail(e, "batch stream");
    if (cap != cudaStreamCaptureStatusNone)
        return fail(STRATA_EINVAL, "engine: a batch without allocation does not run on a capturing stream");
    unsigned char* scratch;
    int rc;
    if ((rc = scratch_address(c->device, &scratch))) return rc;
    int* d_status = reinterpret_cast<int*>(scratch);
    auto* d_items = reinterpret_cast<strata::BatchItem*>(scratch + kScratchHead);
    auto* d_vitems = reinterpret_cast<strata::ValidityItem*>(scratch + kScratchHead + kItemBytes);
    strata::BatchItem* host = g_noalloc_items;
    for (int i = 0; i < nitems; i++) {
        int nout = 0;
        if ((rc = fill_batch_item(c, items[i], i, host[i], &nout))) return rc;
        host[i].p.status = d_status;
    }
    const int nc = strata::batch_plan(host, nitems, g_noalloc_order, g_noalloc_classes, nullptr);
    if (nc < 0) return fail(STRATA_ENOTSUP, "engine: an op of the batch has no batch kernel");
    strata::ValidityClass vcls[STRATA_MAX_RADIUS + 1];
    int nvc = 0;
    const int nv = strata::batch_plan_validity(host, nitems, g_noalloc_vitems, vcls, &nvc);
    // The status word is not cleared here: a status that an unsynchronised
    // call's kernels set stays until a synchronised call reads and clears it.
    e = cudaMemcpyAsync(d_items, host, sizeof(strata::BatchItem) * (size_t)nitems, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nv > 0)
        e = cudaMemcpyAsync(d_vitems, g_noalloc_vitems, sizeof(strata::ValidityItem) * (size_t)nv,
                            cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e, "batch descriptors");
    for (int i = 0; i < nc; i++)
        if (!strata::launch_batch_class(g_noalloc_classes[i], d_items, st))
            return fail(STRATA_ENOTSUP, "engine: an op of the batch has no batch kernel");
    for (int i = 0; i < nvc; i++) strata::launch_batch_validity(vcls[i], d_vitems, st);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "batch launch");
    if (!synchronize) return STRATA_OK;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(e, "batch run");
    int status = 0;
    if ((e = cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "batch status");
    if (status) {
        if ((e = cudaMemset(d_status, 0, sizeof(int))) != cudaSuccess) return cuda_fail(e, "batch status");
        return fail(status, "engine: a batch kernel reported status %d", status);
    }
    return STRATA_OK;
}

// ---------------------------------------------------------------------------
// Serving: window requests over a resident mosaic, admitted under a memory
// budget and batched as they arrive (continuous batching). A scheduler
// thread takes the queued requests whenever one of its streams is free,
// admits them in arrival order while their outputs fit the budget, and
// launches them as one batch (one persistent kernel per op class) on that
// stream; batches on different streams overlap on the device, and a
// request that arrives while others run joins the next batch. Outputs are
// allocated from a stream-ordered pool and count against the budget until
// released.

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Request {
    uint64_t ticket = 0;
    int64_t x = 0, y = 0, w = 0, h = 0;
    std::vector<strata_stage> stages;
    std::vector<std::vector<float>> tables;  // copies of the stages' tables
    LaunchParams p;
    int nout = 0;
    int status = 1;  // 1 queued, 2 running, 0 done, < 0 failed
    void* block = nullptr;  // one pool allocation holding the outputs below
    float* out[2] = {nullptr, nullptr};
    uint32_t* out_bits[2] = {nullptr, nullptr};
    size_t bytes = 0;  // budget charge
    int64_t t_submit = 0, t_start = 0, t_done = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    strata::BatchItem* d_items = nullptr;
    strata::BatchItem* h_items = nullptr;  // page-locked staging
    strata::ValidityItem* d_vitems = nullptr;
    strata::ValidityItem* h_vitems = nullptr;  // page-locked staging
    std::vector<int> order;
    std::vector<strata::BatchClass> classes;
    std::vector<Request*> reqs;
    bool busy = false;
};

}  // namespace

struct strata_server {
    strata_ctx* ctx = nullptr;
    strata_raster mosaic{};
    DevOperand dm;
    size_t budget = 0, used = 0;
    int max_batch = 64;
    int band = 16;  // rows per unit of the radius-1 batch kernels
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv;       // the scheduler waits here
    std::condition_variable done_cv;  // callers waiting for results
    std::deque<Request*> queue;
    std::vector<void*> to_free;  // released requests' allocations, freed by the scheduler
    std::unordered_map<uint64_t, Request*> all;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread thread;
    cudaMemPool_t pool = nullptr;
    int64_t batches = 0, served = 0;
};

namespace {

// Launches one batch of admitted requests on slot s (scheduler thread,
// with the server lock held): each request a raster of the batch, planned
// and run by the batch kernels, its validity alongside.
int launch_batch(strata_server* S, Slot& s) {
    cudaStream_t st = s.stream;
    const int n = (int)s.reqs.size();
    for (int i = 0; i < n; i++) {
        Request* r = s.reqs[(size_t)i];
        strata::BatchItem& b = s.h_items[i];
        memset(&b, 0, sizeof b);
        b.p = r->p;
        if (r->p.radius <= 1) b.th = S->band;
        for (int k = 0; k < r->nout; k++) {
            if (!r->out_bits[k]) continue;
            ValidityParams& v = b.v[b.nvalid++];
            memset(&v, 0, sizeof v);
            if (S->mosaic.valid) {
                v.src_bits = S->dm.bits;
                v.src_off = S->dm.bit_off + r->y * S->dm.stride + r->x;
                v.src_stride = S->dm.stride;
                v.src_lo_word = S->dm.lo_word;
                v.src_hi_word = S->dm.hi_word;
            }
            v.dst_bits = r->out_bits[k];
            v.dst_off = 0;
            v.dst_stride = r->w;
            v.out_x1 = r->w;
            v.out_y1 = r->h;
            v.width = r->w;
            v.height = r->h;
            v.radius = r->p.radius;
            v.dst_words = (r->w * r->h + 31) / 32;
        }
        const LaunchParams& p = b.p;
        b.vec = aligned16_host(p.src) && aligned16_host(p.dst0) && !(p.src_stride & 3) && !(p.dst0_stride & 3) &&
                (r->nout < 2 || (aligned16_host(p.dst1) && !(p.dst1_stride & 3)));
    }
    const int nc = strata::batch_plan(s.h_items, n, s.order.data(), s.classes.data(), nullptr);
    if (nc < 0) return fail(STRATA_ENOTSUP, "engine: an op of the request has no batch kernel");
    strata::ValidityClass vcls[STRATA_MAX_RADIUS + 1];
    int nvc = 0;
    const int nv = strata::batch_plan_validity(s.h_items, n, s.h_vitems, vcls, &nvc);
    cudaError_t e = cudaMemcpyAsync(s.d_items, s.h_items, sizeof(strata::BatchItem) * (size_t)n,
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nv > 0)
        e = cudaMemcpyAsync(s.d_vitems, s.h_vitems, sizeof(strata::ValidityItem) * (size_t)nv, cudaMemcpyHostToDevice,
                            st);
    if (e != cudaSuccess) return cuda_fail(e, "serve descriptors");
    for (int i = 0; i < nc; i++)
        if (!strata::launch_batch_class(s.classes[(size_t)i], s.d_items, st))
            return fail(STRATA_ENOTSUP, "engine: an op of the request has no batch kernel");
    for (int i = 0; i < nvc; i++) strata::launch_batch_validity(vcls[i], s.d_vitems, st);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaEventRecord(s.done, st);
    if (e != cudaSuccess) return cuda_fail(e, "serve launch");
    return STRATA_OK;
}

constexpr int64_t kCoalesceNs = 100000;  // how long a short queue waits for company while a batch runs

void scheduler(strata_server* S) {
    cudaSetDevice(S->ctx->device);
    std::unique_lock<std::mutex> lk(S->mu);
    std::vector<void*> frees;
    while (!S->stop) {
        bool progressed = false;
        // Return released allocations to the pool, without the lock.
        if (!S->to_free.empty()) {
            frees.swap(S->to_free);
            lk.unlock();
            for (void* p : frees) cudaFreeAsync(p, S->ctx->stream);
            frees.clear();
            lk.lock();
            progressed = true;
        }
        // Retire finished batches.
        for (Slot& s : S->slots) {
            if (!s.busy) continue;
            cudaError_t q = cudaEventQuery(s.done);
            if (q == cudaErrorNotReady) continue;
            const int64_t t = now_ns();
            for (Request* r : s.reqs) {
                r->status = q == cudaSuccess ? 0 : STRATA_ECUDA;
                r->t_done = t;
            }
            S->served += (int64_t)s.reqs.size();
            s.reqs.clear();
            s.busy = false;
            progressed = true;
            S->done_cv.notify_all();
        }
        // Admit queued requests onto a free stream, in arrival order, while
        // their outputs fit the budget. While another batch runs, a short
        // queue waits up to kCoalesceNs for more requests to join it, so
        // that batches grow with the load; an idle server launches at once.
        bool running = false;
        for (Slot& s : S->slots) running = running || s.busy;
        const bool hold = running && !S->queue.empty() && (int)S->queue.size() < S->max_batch / 4 &&
                          now_ns() - S->queue.front()->t_submit < kCoalesceNs;
        for (Slot& s : S->slots) {
            if (hold) break;
            if (s.busy || S->queue.empty()) continue;
            while (!S->queue.empty() && (int)s.reqs.size() < S->max_batch) {
                Request* r = S->queue.front();
                if (S->used + r->bytes > S->budget && !(S->used == 0 && s.reqs.empty())) break;
                // Outputs and their validity words from the stream-ordered
                // pool, in one allocation (one call to allocate and one to
                // free per request), each part on a 256-byte boundary.
                const size_t data_bytes = ((size_t)(r->w * r->h) * 4 + 255) & ~(size_t)255;
                const size_t bit_bytes = S->mosaic.valid ? ((size_t)((r->w * r->h + 63) / 64) * 8 + 255) & ~(size_t)255 : 0;
                if (cudaMallocFromPoolAsync(&r->block, (data_bytes + bit_bytes) * (size_t)r->nout, S->pool, s.stream) !=
                    cudaSuccess) {
                    r->block = nullptr;
                    cudaGetLastError();
                    break;
                }
                for (int k = 0; k < r->nout; k++) {
                    char* base = static_cast<char*>(r->block) + (data_bytes + bit_bytes) * (size_t)k;
                    r->out[k] = reinterpret_cast<float*>(base);
                    if (S->mosaic.valid) r->out_bits[k] = reinterpret_cast<uint32_t*>(base + data_bytes);
                }
                S->queue.pop_front();
                S->used += r->bytes;
                r->p.dst0 = r->out[0];
                r->p.dst0_stride = r->w;
                r->p.dst1 = r->out[1];
                r->p.dst1_stride = r->w;
                r->status = 2;
                r->t_start = now_ns();
                s.reqs.push_back(r);
            }
            if (s.reqs.empty()) break;  // the budget holds even one request back
            int rc = launch_batch(S, s);
            if (rc != STRATA_OK) {
                for (Request* r : s.reqs) {
                    r->status = rc;
                    r->t_done = now_ns();
                }
                s.reqs.clear();
                S->done_cv.notify_all();
                continue;
            }
            s.busy = true;
            S->batches++;
            progressed = true;
        }
        if (!progressed) {
            bool any_busy = false;
            for (Slot& s : S->slots) any_busy = any_busy || s.busy;
            // Poll running batches often; sleep until work arrives otherwise.
            if (any_busy) S->cv.wait_for(lk, std::chrono::microseconds(20));
            else S->cv.wait_for(lk, std::chrono::milliseconds(5));
        }
    }
}

}  // namespace

extern "C" int strata_server_create(strata_ctx* c, const strata_raster* mosaic, const strata_server_opts* o,
                                    strata_server** out) {
    if (!c || !mosaic || !out) return fail(STRATA_EINVAL, "engine: nil argument");
    *out = nullptr;
    int rc = validate("src", 0, *mosaic);
    if (rc) return rc;
    if (!mosaic->on_device) return fail(STRATA_EINVAL, "engine: the served mosaic must be on the device");
    auto* S = new strata_server;
    S->ctx = c;
    S->mosaic = *mosaic;
    S->budget = o && o->budget_bytes ? (size_t)o->budget_bytes : (size_t)120 << 30;
    S->max_batch = o && o->max_batch > 0 ? o->max_batch : 64;
    if (o && (o->band < 0 || o->band > 256)) {
        delete S;
        return fail(STRATA_EINVAL, "engine: server band %d (1 to 256, 0 for the default)", o->band);
    }
    S->band = o && o->band > 0 ? o->band : 16;
    const int nstreams = o && o->streams > 0 ? o->streams : 4;
    DeviceGuard device_guard(c->device);
    if ((rc = stage_in(c, nullptr, *mosaic, 0, false, &S->dm))) {
        delete S;
        return rc;
    }
    cudaError_t e = cudaDeviceGetDefaultMemPool(&S->pool, c->device);
    S->slots.resize((size_t)nstreams);
    for (Slot& s : S->slots) {
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&s.d_items, sizeof(strata::BatchItem) * (size_t)S->max_batch);
        if (e == cudaSuccess)
            e = cudaHostAlloc(&s.h_items, sizeof(strata::BatchItem) * (size_t)S->max_batch, cudaHostAllocDefault);
        if (e == cudaSuccess) e = cudaMalloc(&s.d_vitems, sizeof(strata::ValidityItem) * 2 * (size_t)S->max_batch);
        if (e == cudaSuccess)
            e = cudaHostAlloc(&s.h_vitems, sizeof(strata::ValidityItem) * 2 * (size_t)S->max_batch,
                              cudaHostAllocDefault);
        s.order.resize((size_t)S->max_batch);
        s.classes.resize((size_t)S->max_batch);
    }
    if (e != cudaSuccess) {
        strata_server_destroy(S);
        return cuda_fail(e, "server set-up");
    }
    S->thread = std::thread(scheduler, S);
    *out = S;
    return STRATA_OK;
}

namespace {

// A checked, planned request for window (x, y, w, h) of the mosaic, with
// its own copies of the stages and their tables (the caller's may go
// away); nullptr and the failure recorded if the request is invalid.
Request* prepare_request(strata_server* S, const strata_stage* stages, int nstages, int64_t x, int64_t y, int64_t w,
                         int64_t h, int* rc_out) {
    const strata_raster& M = S->mosaic;
    if (w <= 0 || h <= 0 || x < 0 || y < 0 || x + w > M.width || y + h > M.height) {
        *rc_out = fail(STRATA_EINVAL, "raster: window %lld×%lld at (%lld, %lld) outside %lld×%lld raster",
                       (long long)w, (long long)h, (long long)x, (long long)y, (long long)M.width,
                       (long long)M.height);
        return nullptr;
    }
    auto* r = new Request;
    r->x = x;
    r->y = y;
    r->w = w;
    r->h = h;
    r->stages.assign(stages, stages + (nstages > 0 ? nstages : 0));
    for (auto& st : r->stages)
        for (int k = 0; k < 4; k++)
            if (st.table[k] && st.table_len[k] > 0) {
                r->tables.emplace_back(st.table[k], st.table[k] + st.table_len[k]);
                st.table[k] = r->tables.back().data();
            }
    int rc = plan_stages(r->stages.data(), (int)r->stages.size(), r->p, &r->nout);
    if (rc == STRATA_OK && is_pointwise((uint32_t)r->p.op))
        rc = fail(STRATA_ENOTSUP, "engine: a pointwise op alone has no batch kernel");
    if (rc == STRATA_OK && r->p.fit)
        rc = fail(STRATA_ENOTSUP, "engine: Wood's fit (FitRadius > 0) has no batch kernel");
    if (rc) {
        delete r;
        *rc_out = rc;
        return nullptr;
    }
    LaunchParams& p = r->p;
    p.src = S->dm.data + y * S->dm.stride + x;
    p.src_stride = S->dm.stride;
    p.src_w = w;
    p.src_h = h;
    p.width = w;
    p.height = h;
    p.out_x1 = w;
    p.out_y1 = h;
    p.status = S->ctx->d_status;
    // The charge is the request's allocation: each output's cells and its
    // validity words, each rounded up to 256 bytes.
    const size_t data_bytes = ((size_t)(w * h) * 4 + 255) & ~(size_t)255;
    const size_t bit_bytes = M.valid ? ((size_t)((w * h + 63) / 64) * 8 + 255) & ~(size_t)255 : 0;
    r->bytes = (data_bytes + bit_bytes) * (size_t)r->nout;
    *rc_out = STRATA_OK;
    return r;
}

// Queues a prepared request (server lock held) and returns its ticket.
uint64_t enqueue(strata_server* S, Request* r) {
    r->ticket = S->next_ticket++;
    r->t_submit = now_ns();
    S->all[r->ticket] = r;
    S->queue.push_back(r);
    return r->ticket;
}

// Frees a finished request's outputs and its budget (server lock held).
int release_locked(strata_server* S, uint64_t ticket) {
    auto it = S->all.find(ticket);
    if (it == S->all.end()) return fail(STRATA_EINVAL, "engine: unknown ticket %llu", (unsigned long long)ticket);
    Request* r = it->second;
    if (r->status > 0) return fail(STRATA_EINVAL, "engine: request %llu is still running", (unsigned long long)ticket);
    // The scheduler returns the allocation to the pool, off the caller's path.
    if (r->block) {
        S->to_free.push_back(r->block);
        S->cv.notify_one();
    }
    if (r->t_start) S->used -= r->bytes;
    S->all.erase(it);
    delete r;
    return STRATA_OK;
}

// Waits for a request (server lock held by lk) and describes its result.
int wait_locked(strata_server* S, std::unique_lock<std::mutex>& lk, uint64_t ticket, int64_t timeout_ms,
                strata_server_result* res) {
    auto it = S->all.find(ticket);
    if (it == S->all.end()) return fail(STRATA_EINVAL, "engine: unknown ticket %llu", (unsigned long long)ticket);
    Request* r = it->second;
    auto done = [&] { return r->status <= 0; };
    if (timeout_ms < 0) S->done_cv.wait(lk, done);
    else if (!S->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), done))
        return fail(STRATA_ETIMEDOUT, "engine: request %llu is not done", (unsigned long long)ticket);
    if (res) {
        memset(res, 0, sizeof *res);
        res->status = r->status;
        for (int k = 0; k < r->nout; k++) {
            res->out[k].data = r->out[k];
            res->out[k].width = r->w;
            res->out[k].height = r->h;
            res->out[k].stride = r->w;
            res->out[k].valid = reinterpret_cast<uint64_t*>(r->out_bits[k]);
            res->out[k].on_device = 1;
        }
        res->nout = r->nout;
        res->t_submit_ns = r->t_submit;
        res->t_start_ns = r->t_start;
        res->t_done_ns = r->t_done;
    }
    return r->status < 0 ? fail(r->status, "engine: request %llu failed", (unsigned long long)ticket) : STRATA_OK;
}

}  // namespace

extern "C" int strata_server_submit(strata_server* S, const strata_stage* stages, int nstages, int64_t x, int64_t y,
                                    int64_t w, int64_t h, uint64_t* ticket) {
    if (!S || !ticket) return fail(STRATA_EINVAL, "engine: nil server");
    int rc;
    Request* r = prepare_request(S, stages, nstages, x, y, w, h, &rc);
    if (!r) return rc;
    std::lock_guard<std::mutex> lk(S->mu);
    *ticket = enqueue(S, r);
    S->cv.notify_one();
    return STRATA_OK;
}

extern "C" int strata_server_submit_many(strata_server* S, const strata_server_request* reqs, int n,
                                         uint64_t* tickets) {
    if (!S || (n > 0 && (!reqs || !tickets))) return fail(STRATA_EINVAL, "engine: nil server");
    if (n < 0) return fail(STRATA_EINVAL, "engine: %d requests", n);
    std::vector<Request*> prepared((size_t)n);
    for (int i = 0; i < n; i++) {
        int rc;
        const strata_server_request& q = reqs[i];
        prepared[(size_t)i] = prepare_request(S, q.stages, q.nstages, q.x, q.y, q.w, q.h, &rc);
        if (!prepared[(size_t)i]) {
            for (int j = 0; j < i; j++) delete prepared[(size_t)j];
            return rc;
        }
    }
    std::lock_guard<std::mutex> lk(S->mu);
    for (int i = 0; i < n; i++) tickets[i] = enqueue(S, prepared[(size_t)i]);
    S->cv.notify_one();
    return STRATA_OK;
}

extern "C" int strata_server_wait(strata_server* S, uint64_t ticket, int64_t timeout_ms, strata_server_result* res) {
    if (!S) return fail(STRATA_EINVAL, "engine: nil server");
    std::unique_lock<std::mutex> lk(S->mu);
    return wait_locked(S, lk, ticket, timeout_ms, res);
}

extern "C" int strata_server_wait_many(strata_server* S, const uint64_t* tickets, int n, int64_t timeout_ms,
                                       strata_server_result* results) {
    if (!S || (n > 0 && !tickets)) return fail(STRATA_EINVAL, "engine: nil server");
    std::unique_lock<std::mutex> lk(S->mu);
    for (int i = 0; i < n; i++) {
        const int rc = wait_locked(S, lk, tickets[i], timeout_ms, results ? results + i : nullptr);
        if (rc) return rc;
    }
    return STRATA_OK;
}

extern "C" int strata_server_release(strata_server* S, uint64_t ticket) {
    if (!S) return fail(STRATA_EINVAL, "engine: nil server");
    std::lock_guard<std::mutex> lk(S->mu);
    DeviceGuard device_guard(S->ctx->device);
    const int rc = release_locked(S, ticket);
    S->cv.notify_one();
    return rc;
}

extern "C" int strata_server_release_many(strata_server* S, const uint64_t* tickets, int n) {
    if (!S || (n > 0 && !tickets)) return fail(STRATA_EINVAL, "engine: nil server");
    std::lock_guard<std::mutex> lk(S->mu);
    DeviceGuard device_guard(S->ctx->device);
    int rc = STRATA_OK;
    for (int i = 0; i < n && rc == STRATA_OK; i++) rc = release_locked(S, tickets[i]);
    S->cv.notify_one();
    return rc;
}

extern "C" int strata_server_stats(strata_server* S, int64_t* batches, int64_t* served, int64_t* used_bytes) {
    if (!S) return fail(STRATA_EINVAL, "engine: nil server");
    std::lock_guard<std::mutex> lk(S->mu);
    if (batches) *batches = S->batches;
    if (served) *served = S->served;
    if (used_bytes) *used_bytes = (int64_t)S->used;
    return STRATA_OK;
}

extern "C" void strata_server_destroy(strata_server* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv.notify_all();
    }
    if (S->thread.joinable()) S->thread.join();
    DeviceGuard device_guard(S->ctx->device);
    for (Slot& s : S->slots) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        if (s.done) cudaEventDestroy(s.done);
        if (s.d_items) cudaFree(s.d_items);
        if (s.h_items) cudaFreeHost(s.h_items);
        if (s.d_vitems) cudaFree(s.d_vitems);
        if (s.h_vitems) cudaFreeHost(s.h_vitems);
        if (s.stream) cudaStreamDestroy(s.stream);
    }
    cudaStreamSynchronize(S->ctx->stream);
    for (void* p : S->to_free) cudaFree(p);
    for (auto& kv : S->all) {
        Request* r = kv.second;
        if (r->block) cudaFree(r->block);
        delete r;
    }
    delete S;
}
