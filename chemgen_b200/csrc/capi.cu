// C ABI (include/chemgen_b200.h): handles, device tables, launch selection,
// host-pointer pipeline and the reference-compatible wrapper.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/chemgen_b200.h"
#include "dev_mech.cuh"

namespace cg {
cudaError_t launch_getrates_fp64(const DevMech& m, const double* P, const double* T, const double* Y, double* wdot,
                                 int64_t ng, int block, double* scratch, int64_t scratch_blocks, cudaStream_t s);
int fp64_smem_block(int ns, size_t smem_per_sm, size_t smem_per_block, long* pts_per_sm);
size_t fp64_global_slice_bytes(int ns);
int fp64_global_blocks_per_sm();
struct StagedPlan;
cudaError_t staged_prepare(const DevMech& m, const cg_mech_view& v, int device, StagedPlan** out);
void staged_release(StagedPlan* p);
cudaError_t launch_getrates_staged(const StagedPlan* p, const DevMech& m, const double* P, const double* T,
                                   const double* Y, double* wdot, int64_t ng, cudaStream_t s,
                                   const unsigned long long* count = nullptr);

struct MixedPlan;
cudaError_t mixed_prepare(const DevMech& m, const cg_mech_view& v, int device, MixedPlan** out);
void mixed_release(MixedPlan* p);
cudaError_t launch_getrates_mixed(const MixedPlan* p, const DevMech& m, const double* P, const double* T,
                                  const double* Y, double* wdot, int64_t ng, void* scratch, size_t scratch_bytes,
                                  cudaStream_t s);
size_t mixed_workspace_bytes(const MixedPlan* p, int64_t ng);
size_t deriv_workspace_bytes(int ns, int64_t ng);
struct JacPlan;
cudaError_t jac_prepare(const DevMech& m, const cg_mech_view& v, int device, JacPlan** out);
void jac_release(JacPlan* p);
size_t jac_rows_workspace_bytes(const JacPlan* p, const DevMech& m, int64_t ng);
cudaError_t launch_jacobian_rows(const JacPlan* p, const DevMech& m, int precision, const double* P, const double* T,
                                 const double* Y, void* J, int64_t ng, double* scratch, size_t scratch_bytes,
                                 cudaStream_t s);
cudaError_t launch_jacobian(const DevMech& m, int precision, const double* P, const double* T, const double* Y,
                            void* J, int64_t ng, double* scratch, int sm_count, cudaStream_t s);
cudaError_t launch_vjp(const DevMech& m, const double* P, const double* T, const double* Y, const double* G, double* gT,
                       double* gY, double* gP, int64_t ng, double* scratch, int sm_count, cudaStream_t s);
}  // namespace cg

struct chemgen_handle {
    int device = 0;
    uint64_t fingerprint = 0;
    // kernels generated for this exact mechanism (generate_chemistry.py --language cuda)
    chemgen_kernel_fn gen_fn = nullptr;
    unsigned gen_modes = 0;
    int use_generated = 1;
    int gen_version = -1;
    int ns = 0, nr = 0;
    int max_side = 0;               // most species on one side of a reaction
    cg::DevMech m{};
    void* dbuf = nullptr;
    int sm_count = 0;
    int fp64_block = 0;             // 32/64/128: shared-memory state; 0: staged kernel or global scratch
    cg::StagedPlan* staged = nullptr;   // FP64 staged kernel (state on chip) when fp64_block is 0
    cg::JacPlan* jac = nullptr;         // row-owner Jacobian (J written once) when its tile fits
    int64_t fp64_slices = 0;        // persistent blocks of the global variant
    std::mutex mu;
    void* ws = nullptr;             // library-owned scratch
    size_t ws_bytes = 0;
    // host pipeline buffers
    double* iobuf = nullptr;             // device staging of the host-pointer path
    size_t iobuf_doubles = 0;
    static constexpr int kIoStreams = 3;
    cudaStream_t streams[kIoStreams] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev[kIoStreams] = {nullptr, nullptr, nullptr};
    cg::MixedPlan* mixed = nullptr;
    cudaError_t mixed_err = cudaSuccess;
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int status_of(cudaError_t e) {
    if (e == cudaSuccess) return CHEMGEN_OK;
    if (e == cudaErrorMemoryAllocation) return CHEMGEN_ERR_OUT_OF_MEMORY;
    return CHEMGEN_ERR_CUDA;
}

bool aligned8(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

// Registry of generated kernel modules, keyed by blob fingerprint.
struct Registered {
    uint64_t fp;
    int ns, nr;
    unsigned modes;
    chemgen_kernel_fn fn;
};
std::mutex& reg_mu() {
    static std::mutex m;
    return m;
}
std::vector<Registered>& registry() {
    static std::vector<Registered> r;
    return r;
}
int g_reg_version = 0;

uint64_t fnv1a(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= b[i];
        h *= 0x100000001b3ull;
    }
    return h;
}

void refresh_generated(chemgen_handle* h) {
    std::lock_guard<std::mutex> lk(reg_mu());
    if (h->gen_version == g_reg_version) return;
    h->gen_version = g_reg_version;
    for (const Registered& r : registry())
        if (r.fp == h->fingerprint && r.ns == h->ns && r.nr == h->nr) {
            h->gen_fn = r.fn;
            h->gen_modes = r.modes;
        }
}


// Host image of the device tables; offsets are relative to the buffer start.
struct Builder {
    std::vector<unsigned char> buf;
    size_t put(const void* src, size_t bytes) {
        size_t off = (buf.size() + 255) / 256 * 256;
        buf.resize(off + std::max<size_t>(bytes, 1));
        if (bytes) std::memcpy(buf.data() + off, src, bytes);
        return off;
    }
};

int build_tables(const cg_mech_view& v, chemgen_handle* h) {
    using namespace cg;
    const int ns = (int)v.s[CG_S_NS], nr = (int)v.s[CG_S_NR];
    if (ns > 0x3fff) return CHEMGEN_ERR_UNSUPPORTED;
    const double* inv_mw = (const double*)v.a[CG_INV_MW];
    const double* tmid = (const double*)v.a[CG_TMID];
    const double* lo = (const double*)v.a[CG_SMH_LO];
    const double* hi = (const double*)v.a[CG_SMH_HI];
    std::vector<double> thermo((size_t)ns * 16, 0.0);
    for (int k = 0; k < ns; ++k) {
        thermo[16 * k] = tmid[k];
        for (int j = 0; j < 7; ++j) {
            thermo[16 * k + 1 + j] = lo[7 * k + j];
            thermo[16 * k + 8 + j] = hi[7 * k + j];
        }
    }
    const int32_t* flags = (const int32_t*)v.a[CG_FLAGS];
    const int32_t* rp = (const int32_t*)v.a[CG_RPTR];
    const int32_t* pp = (const int32_t*)v.a[CG_PPTR];
    const int32_t* rsp = (const int32_t*)v.a[CG_RSP];
    const int32_t* psp = (const int32_t*)v.a[CG_PSP];
    const double* rnu = (const double*)v.a[CG_RNU];
    const double* pnu = (const double*)v.a[CG_PNU];
    const double* arh = (const double*)v.a[CG_ARH];
    const double* karh = (const double*)v.a[CG_KARH];
    const double* fall = (const double*)v.a[CG_FALL];
    const double* kfall = (const double*)v.a[CG_KFALL];
    std::vector<DRxn> rx(nr);
    // general-stoichiometry rows: reactant entries then product entries
    std::vector<int> rptr{0}, pptr{0}, gsp_r, gsp_p;
    std::vector<double> gnu_r, gnu_p;
    int seg[CG_NKINDS + 1];
    seg[0] = 0;
    for (int k = 0; k < CG_NKINDS; ++k) seg[k + 1] = seg[k] + (int)v.s[CG_S_NSTD + k];
    const int fall0 = seg[CG_LINDEMANN], plog0 = seg[CG_PLOG];
    for (int r = 0; r < nr; ++r) {
        DRxn& R = rx[r];
        std::memset(&R, 0, sizeof(R));
        R.lnA = karh[4 * r];
        R.b = karh[4 * r + 1];
        R.theta = karh[4 * r + 2];
        R.sgn = (arh[3 * r] == 0.0) ? 0.0 : karh[4 * r + 3];
        if (R.sgn == 0.0) R.lnA = 0.0;
        R.flags = flags[r];
        R.gen = -1;
        if (r >= fall0 && r < plog0) R.aux = r - fall0;
        else if (r >= plog0) R.aux = r - plog0;
        const int nre = rp[r + 1] - rp[r], npr = pp[r + 1] - pp[r];
        h->max_side = std::max(h->max_side, std::max(nre, npr));
        bool compact = nre <= kMaxCompact && npr <= kMaxCompact;
        for (int j = rp[r]; compact && j < rp[r + 1]; ++j)
            compact = (rnu[j] == 1.0 || rnu[j] == 2.0 || rnu[j] == 3.0);
        for (int j = pp[r]; compact && j < pp[r + 1]; ++j)
            compact = (pnu[j] == 1.0 || pnu[j] == 2.0 || pnu[j] == 3.0);
        if (compact) {
            R.flags |= kFCompact;
            R.nre = (unsigned char)nre;
            R.npr = (unsigned char)npr;
            for (int j = 0; j < nre; ++j)
                R.sp[j] = (unsigned short)(rsp[rp[r] + j] | ((int)rnu[rp[r] + j] << 14));
            for (int j = 0; j < npr; ++j)
                R.sp[3 + j] = (unsigned short)(psp[pp[r] + j] | ((int)pnu[pp[r] + j] << 14));
        } else {
            R.gen = (int)rptr.size() - 1;
            for (int j = rp[r]; j < rp[r + 1]; ++j) {
                gsp_r.push_back(rsp[j]);
                gnu_r.push_back(rnu[j]);
            }
            for (int j = pp[r]; j < pp[r + 1]; ++j) {
                gsp_p.push_back(psp[j]);
                gnu_p.push_back(pnu[j]);
            }
            rptr.push_back((int)gsp_r.size());
            pptr.push_back((int)gsp_p.size());
        }
    }
    const int ng_rows = (int)rptr.size() - 1;
    // device entry arrays: all reactant entries, then all product entries
    std::vector<int> dev_sp(gsp_r);
    dev_sp.insert(dev_sp.end(), gsp_p.begin(), gsp_p.end());
    std::vector<double> dev_nu(gnu_r);
    dev_nu.insert(dev_nu.end(), gnu_p.begin(), gnu_p.end());
    for (auto& x : pptr) x += (int)gsp_r.size();

    const int nfall = (int)(v.s[CG_S_NLIND] + v.s[CG_S_NTROE] + v.s[CG_S_NSRI]);
    std::vector<DFall> fl(std::max(nfall, 1));
    std::vector<DFall2> fl2(std::max(nfall, 1));
    for (int f = 0; f < nfall; ++f) {
        const double* row = fall + 8 * f;
        DFall& F = fl[f];
        std::memset(&F, 0, sizeof(F));
        F.lnA0 = kfall[4 * f];
        F.b0 = kfall[4 * f + 1];
        F.theta0 = kfall[4 * f + 2];
        F.sgn0 = (row[0] == 0.0) ? 0.0 : kfall[4 * f + 3];
        if (F.sgn0 == 0.0) F.lnA0 = 0.0;
        const int r = fall0 + f;
        fl2[f].T2 = 0.0;
        fl2[f].pad = 0.0;
        if (r >= seg[CG_TROE] && r < seg[CG_TROE + 1]) {
            F.p[0] = row[7];            // 1 - a
            F.p[1] = 1.0 / row[4];      // 1/T3
            F.p[2] = row[3];            // a
            F.p[3] = 1.0 / row[5];      // 1/T1
            fl2[f].T2 = row[6];
        } else if (r >= seg[CG_SRI] && r < seg[CG_SRI + 1]) {
            F.p[0] = row[3];            // a
            F.p[1] = row[4];            // b
            F.p[2] = 1.0 / row[5];      // 1/c
            F.p[3] = row[6];            // d
            fl2[f].T2 = row[7];         // e
        }
    }
    const int nplog = (int)v.s[CG_S_NPLOG], nlev = (int)v.s[CG_S_NPLEV], nterm = (int)v.s[CG_S_NPTERM];
    std::vector<double> term(4 * (size_t)std::max(nterm, 1), 0.0);
    const double* kterm = (const double*)v.a[CG_KPLOG_TERM];
    const double* pterm = (const double*)v.a[CG_PLOG_TERM];
    for (int t = 0; t < nterm; ++t) {
        term[4 * t] = kterm[4 * t];
        term[4 * t + 1] = kterm[4 * t + 1];
        term[4 * t + 2] = kterm[4 * t + 2];
        term[4 * t + 3] = (pterm[3 * t] == 0.0) ? 0.0 : kterm[4 * t + 3];
    }

    Builder b;
    size_t o_inv = b.put(inv_mw, sizeof(double) * ns);
    size_t o_th = b.put(thermo.data(), sizeof(double) * thermo.size());
    size_t o_rx = b.put(rx.data(), sizeof(DRxn) * rx.size());
    size_t o_ep = b.put(v.a[CG_EFF_PTR], sizeof(int32_t) * (nr + 1));
    size_t o_es = b.put(v.a[CG_EFF_SP], sizeof(int32_t) * v.s[CG_S_NEFF]);
    size_t o_ev = b.put(v.a[CG_EFF_VAL], sizeof(double) * v.s[CG_S_NEFF]);
    size_t o_fl = b.put(fl.data(), sizeof(DFall) * fl.size());
    size_t o_fl2 = b.put(fl2.data(), sizeof(DFall2) * fl2.size());
    size_t o_grp = b.put(rptr.data(), sizeof(int) * rptr.size());
    size_t o_gpp = b.put(pptr.data(), sizeof(int) * pptr.size());
    size_t o_gsp = b.put(dev_sp.data(), sizeof(int) * dev_sp.size());
    size_t o_gnu = b.put(dev_nu.data(), sizeof(double) * dev_nu.size());
    size_t o_pp = b.put(v.a[CG_PLOG_PTR], sizeof(int32_t) * (nplog + 1));
    size_t o_plp = b.put(v.a[CG_PLOG_P], sizeof(double) * nlev);
    size_t o_pln = b.put(v.a[CG_PLOG_LNP], sizeof(double) * nlev);
    size_t o_ptp = b.put(v.a[CG_PLOG_TPTR], sizeof(int32_t) * (nlev + 1));
    size_t o_pt = b.put(term.data(), sizeof(double) * term.size());

    void* d = nullptr;
    cudaError_t e = cudaMalloc(&d, b.buf.size());
    if (e != cudaSuccess) return status_of(e);
    e = cudaMemcpy(d, b.buf.data(), b.buf.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(d);
        return status_of(e);
    }
    auto at = [d](size_t off) { return static_cast<char*>(d) + off; };
    DevMech& m = h->m;
    m.ns = ns;
    m.nr = nr;
    for (int k = 0; k <= CG_NKINDS; ++k) m.seg[k] = seg[k];
    m.has_m = (seg[CG_PLOG] - seg[CG_THIRD_BODY]) > 0;
    m.n_general = ng_rows;
    m.inv_mw = (const double*)at(o_inv);
    m.thermo = (const double*)at(o_th);
    m.rxn = (const DRxn*)at(o_rx);
    m.eff_ptr = (const int*)at(o_ep);
    m.eff_sp = (const int*)at(o_es);
    m.eff_val = (const double*)at(o_ev);
    m.fall = (const DFall*)at(o_fl);
    m.fall2 = (const DFall2*)at(o_fl2);
    m.gen_rptr = (const int*)at(o_grp);
    m.gen_pptr = (const int*)at(o_gpp);
    m.gen_sp = (const int*)at(o_gsp);
    m.gen_nu = (const double*)at(o_gnu);
    m.plog_ptr = (const int*)at(o_pp);
    m.plog_p = (const double*)at(o_plp);
    m.plog_lnp = (const double*)at(o_pln);
    m.plog_tptr = (const int*)at(o_ptp);
    m.plog_term = (const double4*)at(o_pt);
    h->dbuf = d;
    h->ns = ns;
    h->nr = nr;
    return CHEMGEN_OK;
}

// Library-owned scratch of at least `bytes`.  The caller holds h->mu.
int ensure_ws_locked(chemgen_handle* h, size_t bytes) {
    if (bytes <= h->ws_bytes) return CHEMGEN_OK;
    if (h->ws) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return status_of(e);
        cudaFree(h->ws);
        h->ws = nullptr;
        h->ws_bytes = 0;
    }
    cudaError_t e = cudaMalloc(&h->ws, bytes);
    if (e != cudaSuccess) {
        h->ws = nullptr;
        return status_of(e);
    }
    h->ws_bytes = bytes;
    return CHEMGEN_OK;
}

size_t fp64_ws_bytes(const chemgen_handle* h, int64_t ng) {
    if (h->fp64_block || h->staged) return 0;
    int64_t chunks = (ng + 63) / 64;
    int64_t slices = std::min<int64_t>(chunks, h->fp64_slices);
    return (size_t)slices * cg::fp64_global_slice_bytes(h->ns);
}

size_t ws_bytes_for(const chemgen_handle* h, int mode, int64_t ng) {
    if (h->use_generated && h->gen_fn && (mode == 0 || mode == 1) && (h->gen_modes & (1u << mode))) return 0;
    if (mode == CHEMGEN_MODE_FP64) return fp64_ws_bytes(h, ng);
    if (mode == CHEMGEN_MODE_MIXED && h->mixed) return cg::mixed_workspace_bytes(h->mixed, ng);
    return 0;
}

int check_args(const chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y,
               const double* w) {
    if (!h || ng < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (ng == 0) return CHEMGEN_OK;
    if (!P || !T || !Y || !w) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (!aligned8(P) || !aligned8(T) || !aligned8(Y) || !aligned8(w)) return CHEMGEN_ERR_MISALIGNED;
    return CHEMGEN_OK;
}

// One launch.  `ws` is scratch the caller provides (may be more or less than
// ws_bytes_for: the FP64 global variant runs as many persistent blocks as
// slices fit, at least one).
int launch(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng, const double* Y, double* w,
           void* ws, size_t ws_bytes, cudaStream_t s) {
    refresh_generated(h);
    if (h->use_generated && h->gen_fn && (mode == CHEMGEN_MODE_FP64 || mode == CHEMGEN_MODE_MIXED) &&
        (h->gen_modes & (1u << mode)))
        return h->gen_fn(mode, P, T, ng, Y, w, s);
    if (mode == CHEMGEN_MODE_FP64) {
        if (!h->fp64_block && h->staged)
            return status_of(cg::launch_getrates_staged(h->staged, h->m, P, T, Y, w, ng, s));
        int64_t slices = 0;
        if (!h->fp64_block) {
            if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255u)) return CHEMGEN_ERR_INVALID_ARGUMENT;
            slices = (int64_t)(ws_bytes / cg::fp64_global_slice_bytes(h->ns));
            if (slices < 1) return CHEMGEN_ERR_INVALID_ARGUMENT;
            slices = std::min<int64_t>(slices, h->fp64_slices);
        }
        return status_of(cg::launch_getrates_fp64(h->m, P, T, Y, w, ng, h->fp64_block, (double*)ws, slices, s));
    }
    if (mode == CHEMGEN_MODE_MIXED) {
        if (!h->mixed) return h->mixed_err == cudaSuccess ? CHEMGEN_ERR_UNSUPPORTED : status_of(h->mixed_err);
        size_t need = cg::mixed_workspace_bytes(h->mixed, ng);
        if (need && (!ws || ws_bytes < need || (reinterpret_cast<uintptr_t>(ws) & 255u)))
            return CHEMGEN_ERR_INVALID_ARGUMENT;
        return status_of(cg::launch_getrates_mixed(h->mixed, h->m, P, T, Y, w, ng, ws, ws_bytes, s));
    }
    return CHEMGEN_ERR_INVALID_ARGUMENT;
}

// Launch with library-owned scratch.
int run_owned(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng, const double* Y,
              double* w, cudaStream_t s) {
    if (mode != CHEMGEN_MODE_FP64 && mode != CHEMGEN_MODE_MIXED) return CHEMGEN_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(h->mu);
    size_t need = ws_bytes_for(h, mode, ng);
    if (need) {
        int st = ensure_ws_locked(h, need);
        if (st) return st;
    }
    return launch(h, mode, P, T, ng, Y, w, h->ws, h->ws_bytes, s);
}

std::mutex g_mu;
chemgen_handle* g_handle = nullptr;

}  // namespace

namespace cg {
// Read-only view of a handle for the other translation units of the library.
const DevMech* handle_mech(const chemgen_handle* h, int* device, int64_t* max_slices) {
    if (device) *device = h->device;
    if (max_slices) *max_slices = h->fp64_slices;
    return &h->m;
}
}  // namespace cg

namespace {
int g_wrapper_status = CHEMGEN_OK;

}  // namespace

extern "C" {

const char* chemgen_version(void) { return "chemgen_b200 1.0 (sm_100a)"; }

const char* chemgen_status_string(int s) {
    switch (s) {
        case CHEMGEN_OK: return "ok";
        case CHEMGEN_ERR_INVALID_ARGUMENT: return "invalid argument";
        case CHEMGEN_ERR_BAD_MECHANISM: return "mechanism blob rejected";
        case CHEMGEN_ERR_CUDA: return "CUDA error";
        case CHEMGEN_ERR_OUT_OF_MEMORY: return "out of device memory";
        case CHEMGEN_ERR_MISALIGNED: return "pointer not 8-byte aligned";
        case CHEMGEN_ERR_UNSUPPORTED: return "mechanism not supported by this path";
        case CHEMGEN_ERR_TOO_LARGE: return "size exceeds a fixed capacity";
        case CHEMGEN_ERR_NO_GLOBAL_MECHANISM: return "no process-wide mechanism installed";
        default: return "unknown status";
    }
}

int chemgen_create(const void* blob, size_t nbytes, int device, chemgen_handle** out) {
    if (!out || !blob) return CHEMGEN_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cg_mech_view v;
    if (cg_mech_parse(blob, nbytes, &v) != 0) return CHEMGEN_ERR_BAD_MECHANISM;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return ndev == 0 ? CHEMGEN_ERR_CUDA : CHEMGEN_ERR_INVALID_ARGUMENT;
    DeviceGuard g(device);
    chemgen_handle* h = new (std::nothrow) chemgen_handle();
    if (!h) return CHEMGEN_ERR_OUT_OF_MEMORY;
    h->device = device;
    h->fingerprint = fnv1a(blob, nbytes);
    int st = build_tables(v, h);
    if (st) {
        delete h;
        return st;
    }
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        cudaFree(h->dbuf);
        delete h;
        return status_of(e);
    }
    h->sm_count = prop.multiProcessorCount;
    long smem_pts = 0;
    h->fp64_block = cg::fp64_smem_block(h->ns, prop.sharedMemPerMultiprocessor, prop.sharedMemPerBlockOptin,
                                        &smem_pts);
    h->fp64_slices = (int64_t)h->sm_count * cg::fp64_global_blocks_per_sm();
    // The staged kernel whenever its tile fits: it is the FP64 kernel when
    // the one-thread-per-point kernel would hold fewer than 8 warps of points
    // per SM in shared memory (state too large for one thread per point to
    // hide its latencies) or none, and it serves the batches whose size is
    // known only on the device (chemgen_getrates_counted).  Beyond it, the
    // global-scratch kernel.
    e = cg::staged_prepare(h->m, v, device, &h->staged);
    if (e == cudaSuccess) {
        if (smem_pts < 256) h->fp64_block = 0;
    } else if (e != cudaErrorNotSupported) {
        cudaFree(h->dbuf);
        delete h;
        return status_of(e);
    }
    e = cg::jac_prepare(h->m, v, device, &h->jac);
    if (e != cudaSuccess && e != cudaErrorNotSupported) {
        if (h->staged) cg::staged_release(h->staged);
        cudaFree(h->dbuf);
        delete h;
        return status_of(e);
    }
    h->mixed_err = cg::mixed_prepare(h->m, v, device, &h->mixed);
    if (h->mixed_err == cudaErrorNotSupported) h->mixed_err = cudaSuccess;
    *out = h;
    return CHEMGEN_OK;
}

int chemgen_destroy(chemgen_handle* h) {
    if (!h) return CHEMGEN_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->device);
    cudaDeviceSynchronize();
    if (h->mixed) cg::mixed_release(h->mixed);
    if (h->staged) cg::staged_release(h->staged);
    if (h->jac) cg::jac_release(h->jac);
    if (h->ws) cudaFree(h->ws);
    if (h->dbuf) cudaFree(h->dbuf);
    if (h->iobuf) cudaFree(h->iobuf);
    for (int i = 0; i < chemgen_handle::kIoStreams; ++i) {
        if (h->streams[i]) cudaStreamDestroy(h->streams[i]);
        if (h->ev[i]) cudaEventDestroy(h->ev[i]);
    }
    delete h;
    return CHEMGEN_OK;
}

int chemgen_num_species(const chemgen_handle* h) { return h ? h->ns : -1; }

int chemgen_register_kernels(uint64_t fingerprint, int ns, int nr, unsigned modes, chemgen_kernel_fn fn) {
    if (!fn || ns <= 0 || nr < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(reg_mu());
    registry().push_back(Registered{fingerprint, ns, nr, modes, fn});
    ++g_reg_version;
    return CHEMGEN_OK;
}

int chemgen_jacobian(chemgen_handle* h, int precision, const double* P, const double* T, int64_t ng,
                     const double* Y, void* J, void* stream) {
    int st = check_args(h, P, T, ng, Y, (const double*)J);
    if (st || ng == 0) return st;
    if (precision != 0 && precision != 1) return CHEMGEN_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->device);
    if (h->max_side > 16) return CHEMGEN_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->jac) {
        st = ensure_ws_locked(h, cg::jac_rows_workspace_bytes(h->jac, h->m, ng));
        if (st) return st;
        return status_of(cg::launch_jacobian_rows(h->jac, h->m, precision, P, T, Y, J, ng, (double*)h->ws,
                                                  h->ws_bytes, (cudaStream_t)stream));
    }
    st = ensure_ws_locked(h, cg::deriv_workspace_bytes(h->ns, ng));
    if (st) return st;
    return status_of(cg::launch_jacobian(h->m, precision, P, T, Y, J, ng, (double*)h->ws, h->sm_count,
                                         (cudaStream_t)stream));
}

int chemgen_getrates_vjp(chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y,
                         const double* G, double* gT, double* gY, double* gP, void* stream) {
    int st = check_args(h, P, T, ng, Y, gY);
    if (st || ng == 0) return st;
    if (!G || !gT || !aligned8(G) || !aligned8(gT) || (gP && !aligned8(gP)))
        return G && gT ? CHEMGEN_ERR_MISALIGNED : CHEMGEN_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->device);
    if (h->max_side > 16) return CHEMGEN_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(h->mu);
    st = ensure_ws_locked(h, cg::deriv_workspace_bytes(h->ns, ng));
    if (st) return st;
    return status_of(cg::launch_vjp(h->m, P, T, Y, G, gT, gY, gP, ng, (double*)h->ws, h->sm_count,
                                    (cudaStream_t)stream));
}

int chemgen_use_generated(chemgen_handle* h, int enable) {
    if (!h) return CHEMGEN_ERR_INVALID_ARGUMENT;
    h->use_generated = enable ? 1 : 0;
    return CHEMGEN_OK;
}

int chemgen_kernel_kind(chemgen_handle* h, int mode) {
    if (!h || (mode != CHEMGEN_MODE_FP64 && mode != CHEMGEN_MODE_MIXED)) return -1;
    refresh_generated(h);
    if (h->use_generated && h->gen_fn && (h->gen_modes & (1u << mode))) return 1;
    if (mode == CHEMGEN_MODE_MIXED && !h->mixed) return -1;
    return 0;
}
int chemgen_num_reactions(const chemgen_handle* h) { return h ? h->nr : -1; }

int chemgen_getrates_ex(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng, const double* Y,
                        double* wdot, void* stream) {
    int st = check_args(h, P, T, ng, Y, wdot);
    if (st || ng == 0) return st;
    DeviceGuard g(h->device);
    return run_owned(h, mode, P, T, ng, Y, wdot, (cudaStream_t)stream);
}

int chemgen_getrates(chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y, double* wdot,
                     void* stream) {
    return chemgen_getrates_ex(h, CHEMGEN_MODE_FP64, P, T, ng, Y, wdot, stream);
}

int chemgen_getrates_counted(chemgen_handle* h, const double* P, const double* T, int64_t ng, const double* Y,
                             double* wdot, const uint64_t* count, void* stream) {
    int st = check_args(h, P, T, ng, Y, wdot);
    if (st || ng == 0) return st;
    if (!count) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(count) & 7u) return CHEMGEN_ERR_MISALIGNED;
    if (!h->staged) return CHEMGEN_ERR_UNSUPPORTED;
    DeviceGuard g(h->device);
    return status_of(cg::launch_getrates_staged(h->staged, h->m, P, T, Y, wdot, ng, (cudaStream_t)stream,
                                                reinterpret_cast<const unsigned long long*>(count)));
}

int chemgen_workspace_bytes(const chemgen_handle* h, int mode, int64_t ng, size_t* bytes) {
    if (!h || !bytes || ng < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (mode == CHEMGEN_MODE_MIXED && !h->mixed) return CHEMGEN_ERR_UNSUPPORTED;
    if (mode != CHEMGEN_MODE_FP64 && mode != CHEMGEN_MODE_MIXED) return CHEMGEN_ERR_INVALID_ARGUMENT;
    *bytes = ws_bytes_for(h, mode, ng);
    return CHEMGEN_OK;
}

int chemgen_getrates_ws(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng, const double* Y,
                        double* wdot, void* workspace, size_t workspace_bytes, void* stream) {
    int st = check_args(h, P, T, ng, Y, wdot);
    if (st || ng == 0) return st;
    DeviceGuard g(h->device);
    return launch(h, mode, P, T, ng, Y, wdot, workspace, workspace_bytes, (cudaStream_t)stream);
}

int chemgen_getrates_host(chemgen_handle* h, int mode, const double* P, const double* T, int64_t ng, const double* Y,
                          double* wdot) {
    if (!h || ng < 0) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (ng == 0) return CHEMGEN_OK;
    if (!P || !T || !Y || !wdot) return CHEMGEN_ERR_INVALID_ARGUMENT;
    if (mode != CHEMGEN_MODE_FP64 && mode != CHEMGEN_MODE_MIXED) return CHEMGEN_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->device);
    const int ns = h->ns;
    // chunks of points: each chunk's Y/wdot are [ns][chunk] slices of the
    // caller's [ns][ng] arrays, copied with one 2D copy each way.  Chunks go
    // round-robin over three streams, so the host-to-device engine can copy
    // chunk c+1 and c+2 while chunk c computes and copies back, and a stream is
    // reused (its in-order queue waiting for chunk c's copy back) only three
    // chunks later: both copy directions stay busy.
    constexpr int NS = chemgen_handle::kIoStreams;
    const int64_t chunk = std::min<int64_t>(ng, std::max<int64_t>(1 << 16, (ng + 15) / 16));
    const size_t per = (size_t)(2 + 2 * ns) * chunk;       // P, T, Y, wdot doubles of one chunk
    std::lock_guard<std::mutex> lk(h->mu);
    cudaError_t e = cudaSuccess;
    if (!h->streams[0]) {
        for (int i = 0; i < NS && e == cudaSuccess; ++i) {
            e = cudaStreamCreateWithFlags(&h->streams[i], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h->ev[i], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) return status_of(e);
    }
    if (h->iobuf_doubles < NS * per) {
        if (h->iobuf) cudaFree(h->iobuf);
        h->iobuf = nullptr;
        h->iobuf_doubles = 0;
        e = cudaMalloc(&h->iobuf, NS * per * sizeof(double));
        if (e != cudaSuccess) return status_of(e);
        h->iobuf_doubles = NS * per;
    }
    int status = CHEMGEN_OK;
    int64_t c = 0;
    for (int64_t i0 = 0; i0 < ng && status == CHEMGEN_OK; i0 += chunk, ++c) {
        const int b = (int)(c % NS);
        cudaStream_t s = h->streams[b];
        const int64_t n = std::min<int64_t>(chunk, ng - i0);
        double* dP = h->iobuf + (size_t)b * per;
        double* dT = dP + chunk;
        double* dY = dT + chunk;
        double* dW = dY + (size_t)ns * chunk;
        e = cudaMemcpyAsync(dP, P + i0, n * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dT, T + i0, n * sizeof(double), cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(dY, n * sizeof(double), Y + i0, ng * sizeof(double), n * sizeof(double), ns,
                                  cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) {
            status = status_of(e);
            break;
        }
        // the chunk's slices are packed with leading dimension n; chunks in
        // flight on different streams share the scratch, so a chunk that
        // needs scratch waits for the previous chunk's kernel
        const size_t need = ws_bytes_for(h, mode, n);
        int st = CHEMGEN_OK;
        if (need) {
            if (need > h->ws_bytes) {
                for (int q = 0; q < NS; ++q) cudaStreamSynchronize(h->streams[q]);
                st = ensure_ws_locked(h, need);
            }
            if (st == CHEMGEN_OK && c > 0) cudaStreamWaitEvent(s, h->ev[(b + NS - 1) % NS], 0);
        }
        if (st == CHEMGEN_OK) st = launch(h, mode, dP, dT, n, dY, dW, h->ws, h->ws_bytes, s);
        if (st) {
            status = st;
            break;
        }
        e = cudaEventRecord(h->ev[b], s);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(wdot + i0, ng * sizeof(double), dW, n * sizeof(double), n * sizeof(double), ns,
                                  cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) status = status_of(e);
    }
    for (int q = 0; q < NS; ++q) {
        const cudaError_t eq = cudaStreamSynchronize(h->streams[q]);
        if (status == CHEMGEN_OK && eq != cudaSuccess) status = status_of(eq);
    }
    return status;
}

int chemgen_init_constants(const void* blob, size_t nbytes) {
    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CHEMGEN_ERR_CUDA;
    chemgen_handle* h = nullptr;
    int st = chemgen_create(blob, nbytes, dev, &h);
    if (st) return st;
    if (g_handle) chemgen_destroy(g_handle);
    g_handle = h;
    return CHEMGEN_OK;
}

int chemgen_free_constants(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_handle) chemgen_destroy(g_handle);
    g_handle = nullptr;
    return CHEMGEN_OK;
}

int chemgen_global_num_species(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return g_handle ? g_handle->ns : -1;
}

int chemgen_init_constants_file(const char* path) {
    if (!path || !*path) path = getenv("CHEMGEN_BLOB");
    if (!path || !*path) path = "getrates.blob";
    FILE* f = fopen(path, "rb");
    if (!f) return CHEMGEN_ERR_INVALID_ARGUMENT;
    std::vector<unsigned char> buf;
    unsigned char tmp[65536];
    size_t n;
    while ((n = fread(tmp, 1, sizeof tmp, f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    const bool bad = ferror(f) != 0;
    fclose(f);
    if (bad || buf.empty()) return CHEMGEN_ERR_INVALID_ARGUMENT;
    return chemgen_init_constants(buf.data(), buf.size());
}

}  // extern "C"

namespace {
// Body shared by the four wrapper symbols: FP64 getrates on the process-wide
// mechanism, synchronous on the legacy default stream.
void wrapper_body(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_c) {
    std::lock_guard<std::mutex> lk(g_mu);
    chemgen_handle* h = g_handle;
    if (!h) {
        g_wrapper_status = CHEMGEN_ERR_NO_GLOBAL_MECHANISM;
        return;
    }
    int st = check_args(h, P, Temp, ng, Ysp, wdot);
    if (st || ng == 0) {
        g_wrapper_status = st;
        return;
    }
    DeviceGuard g(h->device);
    // Large mechanisms keep per-point state in scratch: the caller's log_c
    // (ng*ns doubles) when it holds at least one block's slice, otherwise
    // library-owned scratch.
    if (!h->fp64_block && !h->staged && log_c) {
        uintptr_t a = reinterpret_cast<uintptr_t>(log_c);
        uintptr_t al = (a + 255) & ~(uintptr_t)255;
        size_t bytes = (size_t)ng * h->ns * sizeof(double);
        if (al - a < bytes && bytes - (al - a) >= cg::fp64_global_slice_bytes(h->ns))
            st = launch(h, CHEMGEN_MODE_FP64, P, Temp, ng, Ysp, wdot, reinterpret_cast<void*>(al), bytes - (al - a), 0);
        else
            st = run_owned(h, CHEMGEN_MODE_FP64, P, Temp, ng, Ysp, wdot, 0);
    } else {
        st = run_owned(h, CHEMGEN_MODE_FP64, P, Temp, ng, Ysp, wdot, 0);
    }
    cudaError_t e = cudaDeviceSynchronize();    // synchronous, as hip_v1_cpp.j2:371
    if (st == CHEMGEN_OK && e != cudaSuccess) st = status_of(e);
    g_wrapper_status = st;
}
}  // namespace

extern "C" {

void getrates_hip_wrapper_v1(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c) {
    (void)log_eg;
    wrapper_body(P, Temp, ng, Ysp, wdot, log_c);
}

void getrates_hip_wrapper_v2(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c) {
    (void)log_eg;
    wrapper_body(P, Temp, ng, Ysp, wdot, log_c);
}

void getrates_hip_wrapper_v3(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c) {
    (void)log_eg;
    wrapper_body(P, Temp, ng, Ysp, wdot, log_c);
}

void getrates_hip_wrapper_v4(double* P, double* Temp, int ng, double* Ysp, double* wdot, double* log_eg,
                             double* log_c) {
    (void)log_eg;
    wrapper_body(P, Temp, ng, Ysp, wdot, log_c);
}

void allocate_intermediate_DeviceMemory(int ng) {
    std::lock_guard<std::mutex> lk(g_mu);
    chemgen_handle* h = g_handle;
    if (!h) {
        g_wrapper_status = CHEMGEN_ERR_NO_GLOBAL_MECHANISM;
        return;
    }
    if (ng < 0) {
        g_wrapper_status = CHEMGEN_ERR_INVALID_ARGUMENT;
        return;
    }
    DeviceGuard g(h->device);
    std::lock_guard<std::mutex> hl(h->mu);
    const size_t need = ws_bytes_for(h, CHEMGEN_MODE_FP64, ng);
    g_wrapper_status = need ? ensure_ws_locked(h, need) : CHEMGEN_OK;
}

int chemgen_last_wrapper_status(void) { return g_wrapper_status; }

}  // extern "C"
