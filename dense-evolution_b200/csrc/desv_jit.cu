// Plan-specialised pass kernels: compile a pass's CUDA source with NVRTC for
// sm_100a, load it with the driver API and launch it on the caller's stream.
// NVRTC and the driver are opened with dlopen on first use, so the library
// still loads (and every other entry point works) where they are absent.
// The kernels themselves are written against csrc/jit_pass.cuh, which reuses
// the tile pipeline and the op bodies of the fused interpreter.
#include <dlfcn.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "desv_common.cuh"
#include "tile_pipeline.cuh"

namespace desv {

// ---- the few NVRTC / driver entry points used (public API signatures)
typedef int nvrtcResult_t;
typedef void *nvrtcProgram_t;
typedef int CUresult_t;
typedef void *CUmodule_t;
typedef void *CUfunction_t;
typedef unsigned long long CUdeviceptr_t;

struct JitApi {
    bool tried = false, ok = false, rtc_ok = false;  // ok: NVRTC and the driver; rtc_ok: NVRTC alone
    std::string why, rtc_why;
    nvrtcResult_t (*CreateProgram)(nvrtcProgram_t *, const char *, const char *, int, const char *const *,
                                   const char *const *);
    nvrtcResult_t (*CompileProgram)(nvrtcProgram_t, int, const char *const *);
    nvrtcResult_t (*GetProgramLogSize)(nvrtcProgram_t, size_t *);
    nvrtcResult_t (*GetProgramLog)(nvrtcProgram_t, char *);
    nvrtcResult_t (*GetCUBINSize)(nvrtcProgram_t, size_t *);
    nvrtcResult_t (*GetCUBIN)(nvrtcProgram_t, char *);
    nvrtcResult_t (*DestroyProgram)(nvrtcProgram_t *);
    CUresult_t (*ModuleLoadData)(CUmodule_t *, const void *);
    CUresult_t (*ModuleUnload)(CUmodule_t);
    CUresult_t (*ModuleGetFunction)(CUfunction_t *, CUmodule_t, const char *);
    CUresult_t (*ModuleGetGlobal)(CUdeviceptr_t *, size_t *, CUmodule_t, const char *);
    CUresult_t (*FuncSetAttribute)(CUfunction_t, int, int);
    CUresult_t (*FuncGetAttribute)(int *, int, CUfunction_t);
    CUresult_t (*OccupancyMaxActiveBlocksPerMultiprocessor)(int *, CUfunction_t, int, size_t);
    CUresult_t (*LaunchKernel)(CUfunction_t, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                               void *, void **, void **);
};

static std::mutex g_jit_mu;
static JitApi g_api;

template <class F> static bool sym(void *lib, const char *name, F &f, std::string &why) {
    f = reinterpret_cast<F>(dlsym(lib, name));
    if (!f) why = std::string("missing symbol ") + name;
    return f != nullptr;
}

static const JitApi &api() {
    std::lock_guard<std::mutex> lk(g_jit_mu);
    if (g_api.tried) return g_api;
    g_api.tried = true;
    void *rtc = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!rtc) rtc = dlopen("libnvrtc.so", RTLD_NOW | RTLD_LOCAL);
    if (!rtc) {
        g_api.why = g_api.rtc_why = "libnvrtc not found";
        return g_api;
    }
    std::string &rw = g_api.rtc_why;
    g_api.rtc_ok = sym(rtc, "nvrtcCreateProgram", g_api.CreateProgram, rw) &&
                   sym(rtc, "nvrtcCompileProgram", g_api.CompileProgram, rw) &&
                   sym(rtc, "nvrtcGetProgramLogSize", g_api.GetProgramLogSize, rw) &&
                   sym(rtc, "nvrtcGetProgramLog", g_api.GetProgramLog, rw) &&
                   sym(rtc, "nvrtcGetCUBINSize", g_api.GetCUBINSize, rw) &&
                   sym(rtc, "nvrtcGetCUBIN", g_api.GetCUBIN, rw) &&
                   sym(rtc, "nvrtcDestroyProgram", g_api.DestroyProgram, rw);
    void *drv = dlopen("libcuda.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!g_api.rtc_ok || !drv) {
        g_api.why = !g_api.rtc_ok ? g_api.rtc_why : "libcuda.so.1 not found";
        return g_api;
    }
    std::string &w = g_api.why;
    g_api.ok = sym(drv, "cuModuleLoadData", g_api.ModuleLoadData, w) &&
               sym(drv, "cuModuleUnload", g_api.ModuleUnload, w) &&
               sym(drv, "cuModuleGetFunction", g_api.ModuleGetFunction, w) &&
               sym(drv, "cuModuleGetGlobal_v2", g_api.ModuleGetGlobal, w) &&
               sym(drv, "cuFuncSetAttribute", g_api.FuncSetAttribute, w) &&
               sym(drv, "cuFuncGetAttribute", g_api.FuncGetAttribute, w) &&
               sym(drv, "cuOccupancyMaxActiveBlocksPerMultiprocessor",
                   g_api.OccupancyMaxActiveBlocksPerMultiprocessor, w) &&
               sym(drv, "cuLaunchKernel", g_api.LaunchKernel, w);
    return g_api;
}

// One loaded pass kernel.
struct JitKernel {
    CUmodule_t mod = nullptr;
    CUfunction_t fn = nullptr;
    CUdeviceptr_t status = 0;  // the module's desv_rtc_status word
    int kind = 0, K = 0, nbuf = 0, dtype = 0, blocks_per_sm = 1;
    size_t smem = 0;  // forward: the launch's dynamic shared memory; adjoint: without the accumulators
    int threads = 0;      // rotation passes: threads per CTA
    int param_floats = 0; // rotation passes: floats in the by-value parameter block
};

// kind of a rotation-pass kernel (desv_rot_load)
constexpr int JIT_KIND_ROT = 5;
constexpr int ROT_REG_BITS = 5;     // fewest register slots per stage (rot_pass.cuh: 32 amplitudes per thread)
constexpr int ROT_MAX_PARAM_FLOATS = 7936;  // by-value parameter block <= 31 KiB (limit 32764 bytes)

// padded stage layout of a 2^K tile: one spare amplitude after every 16
static size_t rot_slot_elems(int K) { return ((size_t)1 << K) + ((size_t)1 << (K - 4)); }

// Adjoint passes: at most this many gradient slots per pass and partial-sum
// rows (the bounds of the interpreter k_adjoint_pass).
constexpr int JIT_ADJ_MAX_PARAMS = 1024;
constexpr int JIT_ADJ_MAX_ROWS = 1184;
int grad_reduce(const double *part, int rows, int np, const int32_t *map, double *grad, cudaStream_t st);
int grad_reduce_rows(const double *part, int rows_x, int np, const int32_t *map, double *grad, int nrows,
                     int64_t grad_stride, cudaStream_t st);
size_t adjoint_scratch_bytes(int max_params);

static std::vector<JitKernel *> g_kernels;  // status words of live modules (under g_jit_mu)

static int jit_status_read_clear() {
    std::vector<CUdeviceptr_t> words;
    {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        for (auto *k : g_kernels) words.push_back(k->status);
    }
    int h = 0;
    for (CUdeviceptr_t w : words) {
        int v = 0;
        if (!w || cudaMemcpy(&v, reinterpret_cast<void *>(w), sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
            continue;
        if (v) {
            const int zero = 0;
            cudaMemcpy(reinterpret_cast<void *>(w), &zero, sizeof(int), cudaMemcpyHostToDevice);
        }
        h |= v;
    }
    return h;
}
static const int jit_status_registered = (register_status_reader(&jit_status_read_clear), 0);

// One tiled Pauli pass through a specialised kernel (called by the Pauli-sum
// driver in desv_api.cu for the passes that have one): same grid rule and
// partial-sum layout as the interpreter pass.
int jit_pauli_launch(void *handle, const void *psi, void *out, int dtype, int mode, const TileGeom &g, int want_e,
                     double *part, int *grid_out, cudaStream_t st) {
    auto *k = static_cast<JitKernel *>(handle);
    if (k->kind != 2 + mode) return fail(DESV_EINVAL, "jit Pauli pass: the kernel was compiled for another mode");
    if (dtype != k->dtype || g.K != k->K || g.K - g.L > 8)
        return fail(DESV_EINVAL, "jit Pauli pass: dtype or tile geometry differs from the compiled kernel");
    const uint64_t ntiles = 1ull << (g.n - k->K);
    const uint64_t cap = (uint64_t)sm_count() * k->blocks_per_sm;
    const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
    *grid_out = (int)grid;
    TileGeom gg = g;
    void *args[] = {const_cast<void **>(&psi), &out, &gg, &want_e, &part};
    if (api().LaunchKernel(k->fn, grid, 1, 1, 256, 1, 1, (unsigned)k->smem, st, args, nullptr) != 0)
        return fail(DESV_ECUDA, "jit Pauli pass: launch failed");
    return DESV_OK;
}

// The same for a rows launch (a kernel compiled with per-row coefficient
// symbols): one grid row per state, CTAs per row by the rows grid rule (at
// most 64), the row's coefficients at csym + row * nsym.
int jit_pauli_rows_launch(void *handle, const void *psi, void *out, int dtype, int mode, const TileGeom &g,
                          int want_e, double *part, int *grid_out, int rows, const RowStrides &rs,
                          const double *csym, int nsym, cudaStream_t st) {
    auto *k = static_cast<JitKernel *>(handle);
    if (k->kind != 2 + mode) return fail(DESV_EINVAL, "jit rows Pauli pass: the kernel was compiled for another mode");
    if (dtype != k->dtype || g.K != k->K || g.K - g.L > 8)
        return fail(DESV_EINVAL, "jit rows Pauli pass: dtype or tile geometry differs from the compiled kernel");
    const uint64_t ntiles = 1ull << (g.n - k->K);
    const uint64_t cap = (uint64_t)sm_count() * k->blocks_per_sm;
    int gx = rows_grid_x(ntiles, cap, rows);
    if (gx > 64) gx = 64;
    *grid_out = gx;
    TileGeom gg = g;
    RowStrides r2 = rs;
    void *args[] = {const_cast<void **>(&psi), &out, &gg, &want_e, &part, const_cast<double **>(&csym), &nsym, &r2};
    if (api().LaunchKernel(k->fn, (unsigned)gx, (unsigned)rows, 1, 256, 1, 1, (unsigned)k->smem, st, args, nullptr) !=
        0)
        return fail(DESV_ECUDA, "jit rows Pauli pass: launch failed");
    return DESV_OK;
}

// Compile CUDA source for sm_100a with NVRTC; the log (if any) goes to log.
static int nvrtc_compile(const char *src, const char *include_dir, std::vector<char> &cubin, char *log,
                         size_t loglen) {
    const JitApi &a = api();
    if (!a.rtc_ok) return fail(DESV_EUNSUPPORTED, "jit: " + a.rtc_why);
    nvrtcProgram_t prog = nullptr;
    if (a.CreateProgram(&prog, src, "desv_pass.cu", 0, nullptr, nullptr) != 0)
        return fail(DESV_ECUDA, "nvrtcCreateProgram failed");
    // include_dir: one or more directories separated by ':'
    std::vector<std::string> incs;
    for (const char *p = include_dir; *p;) {
        const char *e = std::strchr(p, ':');
        const size_t len = e ? (size_t)(e - p) : std::strlen(p);
        if (len) incs.push_back(std::string("-I") + std::string(p, len));
        p += len + (e ? 1 : 0);
    }
    // -default-device: the C-ABI prototypes of desv.h parse as (unused) device declarations
    std::vector<const char *> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-default-device"};
    for (auto &i : incs) opts.push_back(i.c_str());
    const int cr = a.CompileProgram(prog, (int)opts.size(), opts.data());
    size_t ls = 0;
    a.GetProgramLogSize(prog, &ls);
    std::string plog(ls, '\0');
    if (ls) a.GetProgramLog(prog, &plog[0]);
    if (log && loglen) {
        std::strncpy(log, plog.c_str(), loglen - 1);
        log[loglen - 1] = 0;
    }
    if (cr != 0) {
        a.DestroyProgram(&prog);
        return fail(DESV_EINVAL, "jit: NVRTC compile failed: " + plog.substr(0, 2000));
    }
    size_t cs = 0;
    a.GetCUBINSize(prog, &cs);
    cubin.resize(cs);
    a.GetCUBIN(prog, cubin.data());
    a.DestroyProgram(&prog);
    return DESV_OK;
}

}  // namespace desv

using namespace desv;

extern "C" int desv_jit_available(char *why, size_t len) {
    const JitApi &a = api();
    if (why && len) {
        std::strncpy(why, a.ok ? "" : a.why.c_str(), len - 1);
        why[len - 1] = 0;
    }
    return a.ok ? 1 : 0;
}

extern "C" int desv_jit_load(const char *src, const char *include_dir, int kind, int tile_bits, int nbuf,
                             int dtype, int device, void **handle, char *log, size_t loglen) {
    if (!src || !include_dir || !handle) return fail(DESV_EINVAL, "jit load: null argument");
    *handle = nullptr;
    if (dtype != DESV_C64 && dtype != DESV_C128) return fail(DESV_EINVAL, "jit load: bad dtype");
    if (kind < 0 || kind > 4)
        return fail(DESV_EINVAL, "jit load: kind must be 0 (pass), 1 (adjoint) or 2..4 (Pauli pass, mode 0..2)");
    if (tile_bits < 9 || tile_bits > (dtype == DESV_C64 ? 13 : 12) || nbuf < 2 || nbuf > 4)
        return fail(DESV_EINVAL, "jit load: bad tile shape");
    if (!api().ok) return fail(DESV_EUNSUPPORTED, "jit: " + api().why);
    std::vector<char> cubin;
    int r = nvrtc_compile(src, include_dir, cubin, log, loglen);
    if (r) return r;
    const JitApi &a = api();
    auto *k = new JitKernel();
    k->kind = kind;
    k->K = tile_bits;
    k->nbuf = nbuf;
    k->dtype = dtype;
    const size_t esz = dtype == DESV_C64 ? 8 : 16;
    const int nw = (1 << (tile_bits - 4)) / 32 > 0 ? (1 << (tile_bits - 4)) / 32 : 1;
    k->smem = PIPE_HDR_BYTES + (size_t)nbuf * (kind == 1 ? 2 : 1) * ((size_t)1 << tile_bits) * esz;
    // adjoint kernels: room for the per-warp gradient accumulators of the largest pass
    const size_t smem_max = k->smem + (kind == 1 ? (size_t)nw * JIT_ADJ_MAX_PARAMS * sizeof(double) : 0);
    size_t ssz = 0;
    // bind the device's primary context to this thread (compiles may run on worker threads)
    if (cudaSetDevice(device) != cudaSuccess) {
        delete k;
        return check_launch("jit load: cudaSetDevice");
    }
    if (a.ModuleLoadData(&k->mod, cubin.data()) != 0 || a.ModuleGetFunction(&k->fn, k->mod, "desv_jit_kernel") != 0 ||
        a.ModuleGetGlobal(&k->status, &ssz, k->mod, "desv_rtc_status") != 0) {
        if (k->mod) a.ModuleUnload(k->mod);
        delete k;
        return fail(DESV_ECUDA, "jit: loading the compiled pass failed (no current CUDA context?)");
    }
    // CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES = 8
    if (a.FuncSetAttribute(k->fn, 8, (int)smem_max) != 0) {
        a.ModuleUnload(k->mod);
        delete k;
        return fail(DESV_ECUDA, "jit: shared-memory attribute refused");
    }
    int b = 0;
    a.OccupancyMaxActiveBlocksPerMultiprocessor(&b, k->fn, kind >= 2 ? 256 : 1 << (tile_bits - 4), k->smem);
    k->blocks_per_sm = b > 0 ? b : 1;
    {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        g_kernels.push_back(k);
    }
    *handle = k;
    return DESV_OK;
}

extern "C" int desv_jit_free(void *handle) {
    if (!handle) return DESV_OK;
    auto *k = static_cast<JitKernel *>(handle);
    {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        for (size_t i = 0; i < g_kernels.size(); ++i)
            if (g_kernels[i] == k) {
                g_kernels.erase(g_kernels.begin() + i);
                break;
            }
    }
    if (api().ok && k->mod) api().ModuleUnload(k->mod);
    delete k;
    return DESV_OK;
}

extern "C" int desv_jit_pass(void *handle, void *sv, int n, int dtype, const desv_pass *ps, const void *mats_dev,
                             void *stream) {
    if (!handle || !sv || !ps || !mats_dev) return fail(DESV_EINVAL, "jit pass: null argument");
    auto *k = static_cast<JitKernel *>(handle);
    if (k->kind != 0) return fail(DESV_EINVAL, "jit pass: the kernel is an adjoint pass");
    if (dtype != k->dtype) return fail(DESV_EINVAL, "jit pass: dtype differs from the compiled kernel");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "jit pass: n out of range");
    if (reinterpret_cast<uintptr_t>(sv) % 16) return fail(DESV_EINVAL, "jit pass: state not 16-byte aligned");
    TileGeom g;
    if (ps->tile_bits != k->K || ps->tile_bits > n || ps->low_bits < 5 || ps->tile_bits - ps->low_bits > 8 ||
        !make_geom(g, n, ps->tile_bits, ps->low_bits, ps->high))
        return fail(DESV_EINVAL, "jit pass: tile geometry does not match the compiled kernel");
    if (ps->op_end == ps->op_begin) return DESV_OK;
    const uint64_t ntiles = 1ull << (n - k->K);
    const uint64_t cap = (uint64_t)sm_count() * k->blocks_per_sm;
    const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
    RowStrides rs{0, 0, 0, 0};
    void *args[] = {&sv, &g, const_cast<void **>(&mats_dev), &rs};
    if (api().LaunchKernel(k->fn, grid, 1, 1, 1u << (k->K - 4), 1, 1, (unsigned)k->smem, stream, args, nullptr) != 0)
        return fail(DESV_ECUDA, "jit pass: launch failed");
    return DESV_OK;
}

extern "C" int desv_jit_pass_rows(void *handle, void *states, int n, int dtype, int rows, const desv_pass *ps,
                                  const void *pools_dev, int64_t pool_stride, void *stream) {
    if (!handle || !states || !ps || !pools_dev) return fail(DESV_EINVAL, "jit rows pass: null argument");
    auto *k = static_cast<JitKernel *>(handle);
    if (k->kind != 0) return fail(DESV_EINVAL, "jit rows pass: the kernel is not a fused pass");
    if (dtype != k->dtype) return fail(DESV_EINVAL, "jit rows pass: dtype differs from the compiled kernel");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "jit rows pass: n out of range");
    if (rows < 1 || rows > 65535) return fail(DESV_EINVAL, "jit rows pass: row count must be in [1, 65535]");
    if (pool_stride < 0) return fail(DESV_EINVAL, "jit rows pass: negative pool stride");
    if (reinterpret_cast<uintptr_t>(states) % 16) return fail(DESV_EINVAL, "jit rows pass: states not 16-byte aligned");
    TileGeom g;
    if (ps->tile_bits != k->K || ps->tile_bits > n || ps->low_bits < 5 || ps->tile_bits - ps->low_bits > 8 ||
        !make_geom(g, n, ps->tile_bits, ps->low_bits, ps->high))
        return fail(DESV_EINVAL, "jit rows pass: tile geometry does not match the compiled kernel");
    if (ps->op_end == ps->op_begin) return DESV_OK;
    const uint64_t ntiles = 1ull << (n - k->K);
    const uint64_t cap = (uint64_t)sm_count() * k->blocks_per_sm;
    const unsigned gx = (unsigned)rows_grid_x(ntiles, cap, rows);
    RowStrides rs{(int64_t)1 << n, pool_stride, 0, 0};
    void *args[] = {&states, &g, const_cast<void **>(&pools_dev), &rs};
    if (api().LaunchKernel(k->fn, gx, (unsigned)rows, 1, 1u << (k->K - 4), 1, 1, (unsigned)k->smem, stream, args,
                           nullptr) != 0)
        return fail(DESV_ECUDA, "jit rows pass: launch failed");
    return DESV_OK;
}

extern "C" int desv_jit_adjoint(void *handle, void *phi, void *lam, int n, int dtype, const desv_adj_pass *ps,
                                const desv_op *ops_dev, const void *mats_dev, const int32_t *map_dev,
                                double *grad_dev, void *scratch, size_t scratch_bytes, void *stream) {
    if (!handle || !phi || !lam || !ps || !ops_dev || !mats_dev || !map_dev || !grad_dev || !scratch)
        return fail(DESV_EINVAL, "jit adjoint: null argument");
    if (phi == lam) return fail(DESV_EINVAL, "jit adjoint: phi and lambda must be distinct buffers");
    auto *k = static_cast<JitKernel *>(handle);
    if (k->kind != 1) return fail(DESV_EINVAL, "jit adjoint: the kernel is not an adjoint pass");
    if (dtype != k->dtype) return fail(DESV_EINVAL, "jit adjoint: dtype differs from the compiled kernel");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "jit adjoint: n out of range");
    if (reinterpret_cast<uintptr_t>(phi) % 16 || reinterpret_cast<uintptr_t>(lam) % 16)
        return fail(DESV_EINVAL, "jit adjoint: states not 16-byte aligned");
    if (ps->nparams < 0 || ps->nparams > JIT_ADJ_MAX_PARAMS || ps->map_begin < 0)
        return fail(DESV_EINVAL, "jit adjoint: parameter range invalid");
    if (scratch_bytes < adjoint_scratch_bytes(ps->nparams)) return fail(DESV_EINVAL, "jit adjoint: scratch too small");
    TileGeom g;
    if (ps->tile_bits != k->K || ps->tile_bits > n || ps->low_bits < 5 || ps->tile_bits - ps->low_bits > 8 ||
        !make_geom(g, n, ps->tile_bits, ps->low_bits, ps->high))
        return fail(DESV_EINVAL, "jit adjoint: tile geometry does not match the compiled kernel");
    if (ps->op_end == ps->op_begin) return DESV_OK;
    const int nw = (1 << (k->K - 4)) / 32 > 0 ? (1 << (k->K - 4)) / 32 : 1;
    const size_t smem = k->smem + (size_t)nw * ps->nparams * sizeof(double);
    int bps = 0;
    api().OccupancyMaxActiveBlocksPerMultiprocessor(&bps, k->fn, 1 << (k->K - 4), smem);
    if (bps < 1) bps = 1;
    const uint64_t ntiles = 1ull << (n - k->K);
    uint64_t cap = (uint64_t)sm_count() * bps;
    if (cap > JIT_ADJ_MAX_ROWS) cap = JIT_ADJ_MAX_ROWS;
    const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
    int np = ps->nparams;
    double *part = static_cast<double *>(scratch);
    RowStrides rs{0, 0, 0, 0};
    const unsigned char *rflag = nullptr;
    int want = 0;
    void *args[] = {&phi, &lam, &g, const_cast<desv_op **>(&ops_dev), const_cast<void **>(&mats_dev), &np, &part, &rs,
                    &rflag, &want};
    if (api().LaunchKernel(k->fn, grid, 1, 1, 1u << (k->K - 4), 1, 1, (unsigned)smem, stream, args, nullptr) != 0)
        return fail(DESV_ECUDA, "jit adjoint: launch failed");
    if (np > 0) return grad_reduce(part, (int)grid, np, map_dev + ps->map_begin, grad_dev, static_cast<cudaStream_t>(stream));
    return DESV_OK;
}

// CTAs per state of a rows adjoint pass (partial-sum rows per state; the
// bound desv_rows_scratch_bytes sizes for)
constexpr int JIT_ADJ_ROWS_X = 64;

extern "C" int desv_jit_adjoint_rows(void *handle, void *phi, void *lam, int n, int dtype, int rows,
                                     const desv_adj_pass *ps, const desv_op *ops_dev, const void *pools_dev,
                                     int64_t pool_stride, const int32_t *map_dev, double *grad_dev,
                                     int64_t grad_stride, void *scratch, size_t scratch_bytes, void *stream) {
    if (!handle || !phi || !lam || !ps || !ops_dev || !pools_dev || !map_dev || !grad_dev || !scratch)
        return fail(DESV_EINVAL, "jit rows adjoint: null argument");
    if (phi == lam) return fail(DESV_EINVAL, "jit rows adjoint: phi and lambda must be distinct buffers");
    auto *k = static_cast<JitKernel *>(handle);
    if (k->kind != 1) return fail(DESV_EINVAL, "jit rows adjoint: the kernel is not an adjoint pass");
    if (dtype != k->dtype) return fail(DESV_EINVAL, "jit rows adjoint: dtype differs from the compiled kernel");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "jit rows adjoint: n out of range");
    if (rows < 1 || rows > 65535) return fail(DESV_EINVAL, "jit rows adjoint: row count must be in [1, 65535]");
    if (pool_stride < 0 || grad_stride < 0) return fail(DESV_EINVAL, "jit rows adjoint: negative stride");
    if (reinterpret_cast<uintptr_t>(phi) % 16 || reinterpret_cast<uintptr_t>(lam) % 16)
        return fail(DESV_EINVAL, "jit rows adjoint: states not 16-byte aligned");
    if (ps->nparams < 0 || ps->nparams > JIT_ADJ_MAX_PARAMS || ps->map_begin < 0)
        return fail(DESV_EINVAL, "jit rows adjoint: parameter range invalid");
    if (scratch_bytes < (size_t)rows * JIT_ADJ_ROWS_X * (size_t)(ps->nparams > 0 ? ps->nparams : 1) * sizeof(double))
        return fail(DESV_EINVAL, "jit rows adjoint: scratch smaller than desv_rows_scratch_bytes(rows, params, 0)");
    TileGeom g;
    if (ps->tile_bits != k->K || ps->tile_bits > n || ps->low_bits < 5 || ps->tile_bits - ps->low_bits > 8 ||
        !make_geom(g, n, ps->tile_bits, ps->low_bits, ps->high))
        return fail(DESV_EINVAL, "jit rows adjoint: tile geometry does not match the compiled kernel");
    if (ps->op_end == ps->op_begin) return DESV_OK;
    const int nw = (1 << (k->K - 4)) / 32 > 0 ? (1 << (k->K - 4)) / 32 : 1;
    const size_t smem = k->smem + (size_t)nw * ps->nparams * sizeof(double);
    int bps = 0;
    api().OccupancyMaxActiveBlocksPerMultiprocessor(&bps, k->fn, 1 << (k->K - 4), smem);
    if (bps < 1) bps = 1;
    const uint64_t ntiles = 1ull << (n - k->K);
    int gx = rows_grid_x(ntiles, (uint64_t)sm_count() * bps, rows);
    if (gx > JIT_ADJ_ROWS_X) gx = JIT_ADJ_ROWS_X;
    int np = ps->nparams;
    double *part = static_cast<double *>(scratch);
    RowStrides rs{(int64_t)1 << n, pool_stride, 0, (int64_t)gx * np};
    const unsigned char *rflag = nullptr;
    int want = 0;
    void *args[] = {&phi, &lam, &g, const_cast<desv_op **>(&ops_dev), const_cast<void **>(&pools_dev), &np, &part,
                    &rs, &rflag, &want};
    if (api().LaunchKernel(k->fn, (unsigned)gx, (unsigned)rows, 1, 1u << (k->K - 4), 1, 1, (unsigned)smem, stream,
                           args, nullptr) != 0)
        return fail(DESV_ECUDA, "jit rows adjoint: launch failed");
    if (np > 0)
        return grad_reduce_rows(part, gx, np, map_dev + ps->map_begin, grad_dev, rows, grad_stride,
                                static_cast<cudaStream_t>(stream));
    return DESV_OK;
}

extern "C" int desv_jit_adjoint_rows_split(void *handle_tangent, void *handle_general, const unsigned char *rflag_dev,
                                           void *phi, void *lam, int n, int dtype, int rows, const desv_adj_pass *ps,
                                           const desv_op *ops_dev, const void *pools_dev, int64_t pool_stride,
                                           const int32_t *map_dev, double *grad_dev, int64_t grad_stride,
                                           void *scratch, size_t scratch_bytes, void *stream) {
    if (!handle_tangent || !handle_general || !rflag_dev || !phi || !lam || !ps || !ops_dev || !pools_dev ||
        !map_dev || !grad_dev || !scratch)
        return fail(DESV_EINVAL, "jit rows adjoint (split): null argument");
    if (phi == lam) return fail(DESV_EINVAL, "jit rows adjoint (split): phi and lambda must be distinct buffers");
    auto *kt = static_cast<JitKernel *>(handle_tangent);
    auto *kg = static_cast<JitKernel *>(handle_general);
    if (kt->kind != 1 || kg->kind != 1) return fail(DESV_EINVAL, "jit rows adjoint (split): not adjoint kernels");
    if (dtype != kt->dtype || dtype != kg->dtype || kt->K != kg->K)
        return fail(DESV_EINVAL, "jit rows adjoint (split): the two kernels differ in dtype or tile width");
    if (n < 1 || n > 34) return fail(DESV_EINVAL, "jit rows adjoint (split): n out of range");
    if (rows < 1 || rows > 65535) return fail(DESV_EINVAL, "jit rows adjoint (split): row count must be in [1, 65535]");
    if (pool_stride < 0 || grad_stride < 0) return fail(DESV_EINVAL, "jit rows adjoint (split): negative stride");
    if (reinterpret_cast<uintptr_t>(phi) % 16 || reinterpret_cast<uintptr_t>(lam) % 16)
        return fail(DESV_EINVAL, "jit rows adjoint (split): states not 16-byte aligned");
    if (ps->nparams < 0 || ps->nparams > JIT_ADJ_MAX_PARAMS || ps->map_begin < 0)
        return fail(DESV_EINVAL, "jit rows adjoint (split): parameter range invalid");
    if (scratch_bytes < (size_t)rows * JIT_ADJ_ROWS_X * (size_t)(ps->nparams > 0 ? ps->nparams : 1) * sizeof(double))
        return fail(DESV_EINVAL, "jit rows adjoint (split): scratch smaller than desv_rows_scratch_bytes");
    TileGeom g;
    if (ps->tile_bits != kt->K || ps->tile_bits > n || ps->low_bits < 5 || ps->tile_bits - ps->low_bits > 8 ||
        !make_geom(g, n, ps->tile_bits, ps->low_bits, ps->high))
        return fail(DESV_EINVAL, "jit rows adjoint (split): tile geometry does not match the compiled kernels");
    if (ps->op_end == ps->op_begin) return DESV_OK;
    const int nw = (1 << (kt->K - 4)) / 32 > 0 ? (1 << (kt->K - 4)) / 32 : 1;
    const size_t smt = kt->smem + (size_t)nw * ps->nparams * sizeof(double);
    const size_t smg = kg->smem + (size_t)nw * ps->nparams * sizeof(double);
    // one grid for both launches (the partial-sum layout the reduction reads):
    // the fewer resident CTAs of the two kernels
    int bt = 0, bg = 0;
    api().OccupancyMaxActiveBlocksPerMultiprocessor(&bt, kt->fn, 1 << (kt->K - 4), smt);
    api().OccupancyMaxActiveBlocksPerMultiprocessor(&bg, kg->fn, 1 << (kg->K - 4), smg);
    int bps = bt < bg ? bt : bg;
    if (bps < 1) bps = 1;
    const uint64_t ntiles = 1ull << (n - kt->K);
    int gx = rows_grid_x(ntiles, (uint64_t)sm_count() * bps, rows);
    if (gx > JIT_ADJ_ROWS_X) gx = JIT_ADJ_ROWS_X;
    int np = ps->nparams;
    double *part = static_cast<double *>(scratch);
    RowStrides rs{(int64_t)1 << n, pool_stride, 0, (int64_t)gx * np};
    for (int want = 1; want >= 0; --want) {
        JitKernel *k = want ? kt : kg;
        int w = want;
        void *args[] = {&phi, &lam, &g, const_cast<desv_op **>(&ops_dev), const_cast<void **>(&pools_dev), &np, &part,
                        &rs, const_cast<unsigned char **>(&rflag_dev), &w};
        if (api().LaunchKernel(k->fn, (unsigned)gx, (unsigned)rows, 1, 1u << (k->K - 4), 1, 1,
                               (unsigned)(want ? smt : smg), stream, args, nullptr) != 0)
            return fail(DESV_ECUDA, "jit rows adjoint (split): launch failed");
    }
    if (np > 0)
        return grad_reduce_rows(part, gx, np, map_dev + ps->map_begin, grad_dev, rows, grad_stride,
                                static_cast<cudaStream_t>(stream));
    return DESV_OK;
}

extern "C" int desv_rot_load(const char *src, const char *include_dirs, int tile_bits, int nbuf, int param_floats,
                             int device, void **handle, char *log, size_t loglen) {
    if (!src || !include_dirs || !handle) return fail(DESV_EINVAL, "rotation pass load: null argument");
    *handle = nullptr;
    if (tile_bits < ROT_REG_BITS + 4 || tile_bits > 12)
        return fail(DESV_EINVAL, "rotation pass load: tile_bits must be in [9, 12]");
    if (nbuf < 1 || nbuf > 3) return fail(DESV_EINVAL, "rotation pass load: nbuf must be 1, 2 or 3");
    if (param_floats < 1 || param_floats > ROT_MAX_PARAM_FLOATS)
        return fail(DESV_EINVAL, "rotation pass load: parameter block size out of range");
    if (!api().ok) return fail(DESV_EUNSUPPORTED, "jit: " + api().why);
    std::vector<char> cubin;
    int r = nvrtc_compile(src, include_dirs, cubin, log, loglen);
    if (r) return r;
    const JitApi &a = api();
    auto *k = new JitKernel();
    k->kind = JIT_KIND_ROT;
    k->K = tile_bits;
    k->nbuf = nbuf;
    k->dtype = DESV_C64;
    k->threads = 0;   // from the kernel's launch bounds once it is loaded (2^(K - register slots))
    k->param_floats = param_floats;
    k->smem = PIPE_HDR_BYTES + (size_t)nbuf * rot_slot_elems(tile_bits) * sizeof(float2);
    size_t ssz = 0;
    if (cudaSetDevice(device) != cudaSuccess) {
        delete k;
        return check_launch("rotation pass load: cudaSetDevice");
    }
    if (a.ModuleLoadData(&k->mod, cubin.data()) != 0 || a.ModuleGetFunction(&k->fn, k->mod, "desv_rot_kernel") != 0 ||
        a.ModuleGetGlobal(&k->status, &ssz, k->mod, "desv_rtc_status") != 0) {
        if (k->mod) a.ModuleUnload(k->mod);
        delete k;
        return fail(DESV_ECUDA, "rotation pass load: loading the compiled pass failed (no current CUDA context?)");
    }
    if (a.FuncSetAttribute(k->fn, 8, (int)k->smem) != 0) {
        a.ModuleUnload(k->mod);
        delete k;
        return fail(DESV_ECUDA, "rotation pass load: shared-memory attribute refused");
    }
    // the generated kernel declares its block size (2^(K - register slots per
    // stage)) in its launch bounds: CU_FUNC_ATTRIBUTE_MAX_THREADS_PER_BLOCK
    int maxt = 0;
    if (a.FuncGetAttribute(&maxt, 0, k->fn) != 0 || maxt < 32 || maxt > (1 << (tile_bits - ROT_REG_BITS)) ||
        (maxt & (maxt - 1))) {
        a.ModuleUnload(k->mod);
        delete k;
        return fail(DESV_EINVAL, "rotation pass load: the kernel's launch bounds are not a block of 2^(K - slots)");
    }
    k->threads = maxt;
    int b = 0;
    a.OccupancyMaxActiveBlocksPerMultiprocessor(&b, k->fn, k->threads, k->smem);
    k->blocks_per_sm = b > 0 ? b : 1;
    {
        std::lock_guard<std::mutex> lk(g_jit_mu);
        g_kernels.push_back(k);
    }
    *handle = k;
    return DESV_OK;
}

extern "C" int desv_rot_pass(void *handle, void *sv, int n, const desv_pass *ps, const float *params,
                             int param_floats, void *stream) {
    if (!handle || !sv || !ps || !params) return fail(DESV_EINVAL, "rotation pass: null argument");
    auto *k = static_cast<JitKernel *>(handle);
    if (k->kind != JIT_KIND_ROT) return fail(DESV_EINVAL, "rotation pass: the kernel is not a rotation pass");
    if (param_floats != k->param_floats)
        return fail(DESV_EINVAL, "rotation pass: parameter block size differs from the compiled kernel's");
    if (n < k->K || n > 34) return fail(DESV_EINVAL, "rotation pass: n out of range");
    if (reinterpret_cast<uintptr_t>(sv) % 16) return fail(DESV_EINVAL, "rotation pass: state not 16-byte aligned");
    TileGeom g;
    if (ps->tile_bits != k->K || ps->low_bits < 5 || ps->tile_bits - ps->low_bits > 8 ||
        !make_geom(g, n, ps->tile_bits, ps->low_bits, ps->high))
        return fail(DESV_EINVAL, "rotation pass: tile geometry does not match the compiled kernel");
    const uint64_t ntiles = 1ull << (n - k->K);
    const uint64_t cap = (uint64_t)sm_count() * k->blocks_per_sm;
    const unsigned grid = (unsigned)(ntiles < cap ? ntiles : cap);
    // the parameter block is the kernel's third (by-value) argument: the
    // launch copies it, so the caller's buffer is free again on return
    void *args[] = {&sv, &g, const_cast<float *>(params)};
    if (api().LaunchKernel(k->fn, grid, 1, 1, (unsigned)k->threads, 1, 1, (unsigned)k->smem, stream, args, nullptr) !=
        0)
        return fail(DESV_ECUDA, "rotation pass: launch failed");
    return DESV_OK;
}

extern "C" int desv_jit_compile_check(const char *src, const char *include_dirs, char *log, size_t loglen) {
    if (!src || !include_dirs) return fail(DESV_EINVAL, "jit compile check: null argument");
    if (!api().rtc_ok) return fail(DESV_EUNSUPPORTED, "jit: " + api().rtc_why);
    std::vector<char> cubin;
    return nvrtc_compile(src, include_dirs, cubin, log, loglen);
}
