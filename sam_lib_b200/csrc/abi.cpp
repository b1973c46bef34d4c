// C ABI of the GPU numeric phase: the SPR entry points a Fortran-77 host
// calls (SPRSOL/SPRFC1/SPRFS1/SPRBS1 with gfortran naming: lower case plus a
// trailing underscore, every argument by reference) and a device-level API.
//
// Integer width: SPR_INT is int64_t for the default INTEGER*8 build
// (-fdefault-integer-8, src/SPR/CMakeLists.txt:12-29) and int32_t for the
// I4 build; the same source is compiled once per width.
//
// Ownership follows SPR: the caller owns every array; the library keeps one
// device context per (MSPAR, MTREES, MSIFA) triple (plan + device buffers),
// and remembers which host SM its device factor came from, so a factorisation
// followed by solves on the same, unmodified SM reuses the device-resident
// factor.  The factor is always written back into SM, so host-only consumers
// of the factor keep working.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "elements.h"
#include "engine.h"
#include "smhash.h"

#ifndef SPR_INT
#define SPR_INT int64_t
#endif
typedef SPR_INT I;

#ifndef SPR_SUFFIX
#define SPR_SUFFIX
#endif
#define SPR_CAT2(a, b) a##b
#define SPR_CAT(a, b) SPR_CAT2(a, b)
#define SPR_API(name) SPR_CAT(name, SPR_SUFFIX)

namespace {

using sprb::Engine;
using sprb::FactorResult;

struct Ctx {
    Engine eng;
    std::vector<int64_t> mspar_snap;   // structure fingerprint (MSPAR without state slots)
    uint64_t tree_hash = 0;
    double* d_sm = nullptr;
    double* d_b = nullptr;
    int64_t b_cap = 0;
    double* d_dcor = nullptr;          // SPRFC3's DCOR(2,NEQ) on the device
    bool dev_chol = false;             // the device holds the L D L' form of a host C C' factor
    cudaStream_t stream = nullptr;
    cudaStream_t copy = nullptr;       // host <-> device copies of a streamed factorisation
    bool streamed_pending = false;     // its timing is read once the copies are done
    // device factor residency
    const double* sm_host = nullptr;
    uint64_t sm_fp = 0;
    bool resident = false;
    ~Ctx() {
        if (d_sm) cudaFree(d_sm);
        if (d_b) cudaFree(d_b);
        if (d_dcor) cudaFree(d_dcor);
        if (stream) cudaStreamDestroy(stream);
        if (copy) cudaStreamDestroy(copy);
    }
};

std::mutex g_mu;
std::map<std::tuple<const void*, const void*, const void*>, std::unique_ptr<Ctx>> g_ctx;

uint64_t mix(uint64_t h, uint64_t v) {
    h ^= v + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    return h;
}

// Residency of the device factor across calls: a solve call reuses the
// device factor only if the host SM still holds exactly what the
// factorisation wrote back.  The check hashes all of the host SM (smhash.h;
// the factorisation hashed the same bytes on the device before the copy), so
// an edit of a single entry between SPRFC1 and SPRFS1 makes the solve
// re-upload SM.  SPR_B200_TRUST_SM=1 skips the host hash: the caller then
// promises not to modify SM between a factorisation and its solves.
bool trust_sm() {
    static const bool t = [] {
        const char* v = std::getenv("SPR_B200_TRUST_SM");
        return v != nullptr && v[0] == '1';
    }();
    return t;
}

int host_threads() {
    const unsigned n = std::thread::hardware_concurrency();
    return (int)std::min(16u, std::max(1u, n));
}

std::vector<int64_t> widen(const I* a, int64_t n) {
    std::vector<int64_t> v(n);
    for (int64_t i = 0; i < n; ++i) v[i] = (int64_t)a[i];
    return v;
}

void msg(I lpu, const char* routine, const char* text) {
    if (lpu < 0) return;
    fprintf(stderr, " *** ERROR return from SPR routine %s (GPU)\n     %s\n", routine, text);
}

// Message of a failed solve: rc -5 is the refused LDB < NEQ layout (see
// reduced_rows_retained), anything else a CUDA failure.
void solve_msg(I lpu, const char* routine, int rc, const char* text) {
    msg(lpu, routine, rc == -5 ? "LDB < NEQ, BUT AN EQUATION OUTSIDE THE RETAINED SUPERNODES IS NUMBERED BEYOND LDB"
                               : text);
}

// Structure fingerprint: MSPAR slots that describe the symbolic structure
// plus a sample of the tree arrays.
void structure_key(const I* mspar, const I* mtrees, const I* msifa, std::vector<int64_t>& snap,
                   uint64_t& h) {
    snap.clear();
    for (int i = 2; i < 25; ++i) snap.push_back((int64_t)mspar[i]);
    for (int i = 40; i < 50; ++i) snap.push_back((int64_t)mspar[i]);
    snap.push_back((int64_t)mspar[56]);              // MSPAR(57): partial factorisation
    h = 0;
    const int64_t nsuper = mspar[10];
    const I* xs = mtrees + (mspar[44] - 1);
    for (int64_t i = 0; i < 3 * (nsuper + 1) - 1; i += 1 + nsuper / 64) h = mix(h, (uint64_t)xs[i]);
    const I* xl = msifa + (mspar[47] - 1);
    for (int64_t i = 0; i <= nsuper; i += 1 + nsuper / 64) h = mix(h, (uint64_t)xl[i]);
}

// Returns the context for this structure (building it when needed) or null.
Ctx* get_ctx(I* mspar, I* mtrees, I* msifa, int& err) {
    err = 0;
    std::vector<int64_t> snap;
    uint64_t h;
    structure_key(mspar, mtrees, msifa, snap, h);
    auto key = std::make_tuple((const void*)mspar, (const void*)mtrees, (const void*)msifa);
    auto it = g_ctx.find(key);
    if (it != g_ctx.end() && it->second->mspar_snap == snap && it->second->tree_hash == h) return it->second.get();
    if (it != g_ctx.end()) g_ctx.erase(it);
    std::unique_ptr<Ctx> c(new Ctx());
    const int64_t nspar = 60;
    std::vector<int64_t> ms(nspar, 0);
    for (int i = 0; i < 58; ++i) ms[i] = (int64_t)mspar[i];
    const int64_t ntrees = mspar[3], nmsifa = mspar[2];
    std::vector<int64_t> mt = widen(mtrees, ntrees), mf = widen(msifa, nmsifa);
    int rc = c->eng.open(ms.data(), mt.data(), mf.data());
    if (rc != 0) {
        err = rc;
        return nullptr;
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        err = -4;
        return nullptr;
    }
    c->eng.set_stream(c->stream);
    const int64_t nsm = mspar[7] + mspar[15];
    if (cudaMalloc((void**)&c->d_sm, nsm * sizeof(double)) != cudaSuccess) {
        err = -4;
        return nullptr;
    }
    c->mspar_snap = snap;
    c->tree_hash = h;
    Ctx* raw = c.get();
    g_ctx[key] = std::move(c);
    return raw;
}

// MVMULT/MMMULT callbacks.  SPRFC1 and SPRFC3 take the LDL' kernels LMVY18
// (y += sum_j (-a_j(1) d_j) a_j, lmvy18.f:5-173) and LMMY18 (packed lower
// Y -= X D X', lmmy18.f:5-192); SPRFC2 takes the C C' kernels CMVY18 and
// CMMY18 (the same without D, cmvy18.f:5, cmmy18.f:5).  The GPU applies the
// update those kernels define and never calls the routine it is given, so a
// routine that computes something else would be ignored silently.  Instead,
// a non-null routine is run once on a small probe (3x3 / 3x2 operands, the
// reference's argument conventions) and the call is refused (IERR = -4)
// unless it reproduces that update.  The outcome is cached per routine.
typedef void (*LmvFn)(I*, I*, double*, double*, I*, double*);
typedef void (*LmmFn)(I*, I*, I*, I*, double*, double*, double*, I*);
typedef void (*CmvFn)(I*, I*, double*, I*, double*);
typedef void (*CmmFn)(I*, I*, I*, I*, double*, double*, I*);

bool close_vec(const double* a, const double* b, int n) {
    for (int i = 0; i < n; ++i)
        if (!(std::fabs(a[i] - b[i]) <= 1e-12 * (1.0 + std::fabs(b[i])))) return false;
    return true;
}

bool probe_mv(void (*f)(), bool with_d) {
    I m = 3, n = 3;
    double A[9] = {0.5, -1.25, 0.75, 1.5, 0.25, -0.5, -0.625, 2.0, 1.125};
    double D[3] = {2.0, -3.0, 0.5};
    I apnt[4] = {1, 4, 7, 10};        // APNT(J+1) - (M+1) = (J-1) M, lmvy18.f:148-150
    double Y[3] = {1.0, -2.0, 0.25}, E[3] = {1.0, -2.0, 0.25};
    for (int j = 0; j < 3; ++j) {
        const double a = -A[3 * j] * (with_d ? D[j] : 1.0);
        for (int i = 0; i < 3; ++i) E[i] += a * A[3 * j + i];
    }
    if (with_d)
        reinterpret_cast<LmvFn>(f)(&m, &n, Y, D, apnt, A);
    else
        reinterpret_cast<CmvFn>(f)(&m, &n, Y, apnt, A);
    return close_vec(Y, E, 3);
}

bool probe_mm(void (*f)(), bool with_d) {
    I m = 3, n = 2, q = 2, ldy = 3;
    double X[6] = {0.5, -1.25, 0.75, 1.5, 0.25, -0.5};
    double D[2] = {2.0, -3.0};
    I xpnt[3] = {1, 4, 7};            // XPNT(J+1) = one past column J, lmmy18.f:18-19
    double Y[5] = {1.0, -2.0, 0.25, 0.5, 3.0}, E[5];
    std::memcpy(E, Y, sizeof(E));
    for (int c = 0, base = 0; c < 2; base += 3 - c, ++c)
        for (int r = c; r < 3; ++r)
            for (int j = 0; j < 2; ++j) E[base + r - c] += -X[3 * j + c] * (with_d ? D[j] : 1.0) * X[3 * j + r];
    if (with_d)
        reinterpret_cast<LmmFn>(f)(&m, &n, &q, xpnt, X, D, Y, &ldy);
    else
        reinterpret_cast<CmmFn>(f)(&m, &n, &q, xpnt, X, Y, &ldy);
    return close_vec(Y, E, 5);
}

// true when both callbacks are null or compute the kernels' update
bool callbacks_ok(void (*mv)(), void (*mm)(), bool ldlt) {
    static std::map<std::pair<const void*, int>, bool> seen;   // under g_mu
    auto check = [&](void (*f)(), int kind) {
        if (!f) return true;
        const auto key = std::make_pair((const void*)f, kind);
        auto it = seen.find(key);
        if (it != seen.end()) return it->second;
        const bool ok = (kind & 1) ? probe_mm(f, (kind & 2) != 0) : probe_mv(f, (kind & 2) != 0);
        seen[key] = ok;
        return ok;
    };
    const int d = ldlt ? 2 : 0;
    return check(mv, d) && check(mm, d | 1);
}

// Reference length checks of SPRFC1 (src/SPR/sprfc1.f:150-236).
bool fc1_lengths_ok(const I* mspar) {
    const int64_t neq = mspar[7], nsuper = mspar[10], nb = mspar[11], mfront = mspar[13];
    const int64_t nofsub = mspar[14], nzerol = mspar[15], wstack = mspar[16], nelact = mspar[18];
    const int64_t nblock = mspar[21], nmsifa = mspar[2], ntrees = mspar[3];
    const int64_t niwork = mfront + 1, nrwork = wstack, nsm = neq + nzerol;
    const int64_t iwused = mfront + 1;
    const int64_t xsuper = mspar[44], xlindx = mspar[45];
    const int64_t supsup = xlindx + nsuper + 1, elseq = supsup + nsuper, xelseq = elseq + nelact;
    const int64_t xblock = xelseq + nb + 1, mtused = xblock + nb;
    (void)xsuper;
    const int64_t lindx = mspar[46], xlnz = mspar[47];
    (void)lindx;
    const int64_t xsplit = xlnz + nsuper + 1, split = xsplit + nsuper, mlused = split + nblock;
    const int64_t smused = neq + nzerol, rwused = wstack;
    (void)nofsub;
    return !(iwused > niwork || mtused > ntrees || mlused > nmsifa || smused > nsm || rwused > nrwork);
}

// Reference length checks of the solves (src/SPR/sprfs1.f:147-226,
// sprbs1.f:141-215; SPRFS2/SPRBS2 the same): MTREES and MSIFA must hold what
// MSPAR says they hold, and LDB >= NEQ (NEQ = LDB when MSPAR(57) = 1).
bool solve_lengths_ok(const I* mspar, I ldb) {
    const int64_t nsuper = mspar[10], nb = mspar[11], nofsub = mspar[14], nelact = mspar[18];
    const int64_t nmsifa = mspar[2], ntrees = mspar[3];
    const int64_t supsup = mspar[45] + nsuper + 1, elseq = supsup + nsuper, xelseq = elseq + nelact;
    const int64_t mtused = xelseq + nb + 1 + nb;
    const int64_t mlused = mspar[46] + nofsub - 1;
    int64_t neq = mspar[7];
    if (mspar[56] == 1 && ldb < neq) neq = ldb;   // sprfs1.f:201
    return !(mtused > ntrees || mlused > nmsifa || ldb < neq);
}

int ensure_b(Ctx* c, int64_t n) {
    if (c->b_cap >= n) return 0;
    if (c->d_b) cudaFree(c->d_b);
    c->d_b = nullptr;
    c->b_cap = 0;
    if (cudaMalloc((void**)&c->d_b, n * sizeof(double)) != cudaSuccess) return -4;
    c->b_cap = n;
    return 0;
}

// A solve with LDB < NEQ (MSPAR(57) = 1) handles only the equations whose
// external number is at most LDB: the reference's gather reads the others as
// zero and its scatter drops them, in every supernode it visits (SPRFB1/
// SPRFB2, SPRFB3/SPRFB4 with PERI2E, sprfs1.f:704-900; SPRBS1 likewise).
// The GPU sweeps run over all equations and zero those rows between the
// forward and the back sweep, which is the same only when every such row
// belongs to a retained supernode (never eliminated, skipped by both
// sweeps), the layout the superelement partition produces.  Anything else
// is refused rather than solved differently.
bool reduced_rows_retained(Ctx* c, const I* msifa, int64_t ldb, bool peri2e) {
    const sprb::Plan& P = c->eng.plan();
    for (int64_t js = 0; js < P.nsuper; ++js) {
        if (P.retained[js]) continue;
        for (int64_t r = P.fst[js]; r < P.fst[js] + P.S[js]; ++r) {
            const int64_t ext = peri2e ? (int64_t)msifa[r] - 1 : r;
            if (ext >= ldb) return false;
        }
    }
    return true;
}

// H2D of SM, device factorisation, D2H of SM.  Returns the SPRFC1 IERR, with
// dcor (host DCOR(2,NEQ)) the SPRFC3 one, with chol the SPRFC2 one (the host
// receives C C', the device keeps its L D L' form for the solves).
// True when the host array lies in page-locked memory (cudaMallocHost,
// cudaHostRegister or a pinned torch tensor): copies from and to it are
// asynchronous DMA, so they can overlap the factorisation.
void trace_start() { sprb::trace_reset(); }
void trace(const char* what) { sprb::trace_point(what); }

bool is_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// The copy stream's downloads of a streamed factorisation must be complete
// before the caller reads SM.
double g_copy_ms[3] = {0.0, 0.0, 0.0};            // of the last streamed factorisation

int finish_copies(Ctx* c) {
    if (!c || !c->copy) return 0;
    if (cudaStreamSynchronize(c->copy) != cudaSuccess) return -4;
    if (c->streamed_pending) {
        c->eng.streamed_times(g_copy_ms);
        c->streamed_pending = false;
    }
    return 0;
}

// defer: leave the streamed factorisation's last downloads running (the
// caller queues a solve behind them and then calls finish_copies).
I do_factor(Ctx* c, I* mspar, double* sm, double* tol, I lpu, double* dcor = nullptr, bool chol = false,
            bool defer = false) {
    const int64_t neq = mspar[7], nzerol = mspar[15];
    const int64_t nsm = neq + nzerol;
    const bool fc4 = chol && dcor;                    // SPRFC4: Cholesky with pivot replacement
    const char* who = fc4 ? "SPRFC4" : chol ? "SPRFC2" : dcor ? "SPRFC3" : "SPRFC1";
    cudaStream_t s = c->stream;
    // SPRFC1 on a pinned SM: upload, factorisation and download overlap, level by level
    const bool streamed = !chol && !dcor && is_pinned(sm);
    if (streamed && !c->copy && cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking) != cudaSuccess) return -4;
    if (!streamed && cudaMemcpyAsync(c->d_sm, sm, nsm * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return -4;
    Engine::Singular fc3{0.0, nullptr};
    if (dcor) {
        if (!c->d_dcor && cudaMalloc((void**)&c->d_dcor, 2 * std::max<int64_t>(neq, 1) * sizeof(double)) != cudaSuccess)
            return -4;
        fc3.tol4 = tol[3];
        fc3.d_dcor = c->d_dcor;
    }
    FactorResult r;
    if (streamed) c->streamed_pending = true;
    trace(streamed ? "factorisation (streamed copies) starts" : "factorisation starts");
    const int frc = streamed ? c->eng.factor_streamed(sm, c->d_sm, tol[0], r, c->copy)
                    : chol   ? c->eng.factor_chol(c->d_sm, tol[0], r, fc4 ? &fc3 : nullptr)
                             : c->eng.factor(c->d_sm, tol[0], r, dcor ? &fc3 : nullptr);
    trace("factorisation returned");
    if (frc != 0) {
        finish_copies(c);
        msg(lpu, who, "CUDA failure in the factorisation");
        return -4;
    }
    const bool chol_ok = chol && (r.lierr == 0 || (fc4 && r.lierr == -33));
    if (chol_ok && c->eng.chol_convert(c->d_sm, true) != 0) return -4;
    uint64_t fp = 0;                                  // hash of exactly what the host receives
    if (c->eng.hash(c->d_sm, nsm, fp) != 0) return -4;
    trace("factor hashed");
    if (streamed) {
        if (!defer && finish_copies(c) != 0) return -4;
    } else if (cudaMemcpyAsync(sm, c->d_sm, nsm * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) {
        return -4;
    }
    if (chol_ok && c->eng.chol_convert(c->d_sm, false) != 0) return -4;
    c->dev_chol = chol_ok;
    if (dcor && cudaMemcpyAsync(dcor, c->d_dcor, 2 * neq * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return -4;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -4;
    I ierr = 0;
    tol[1] = r.tol2;
    tol[2] = r.tol3;
    if (r.lierr == -31 || r.lierr == -33) {           // sprfc3.f:249-258, sprfc4.f:244-256
        ierr = -3;
        mspar[26] = -(I)r.supeqt;
        if (lpu >= 0) {
            char buf[256];
            snprintf(buf, sizeof buf, "SINGULAR EQUATION SYSTEM: %" PRId64 " PIVOT(S) REPLACED (TOL(1) = %g)",
                     r.supeqt, tol[0]);
            msg(lpu, who, buf);
        }
        c->sm_host = sm;
        c->sm_fp = fp;
        c->resident = true;
    } else if (r.lierr != 0) {                        // sprfc1.f:251-265
        ierr = (r.lierr / 10 == -3) ? -3 : -4;
        mspar[26] = (I)r.supeqt;
        if (lpu >= 0) {
            char buf[256];
            if (r.lierr == -35)
                snprintf(buf, sizeof buf, "SINGULAR EQUATION SYSTEM: %" PRId64 " ZERO PIVOT(S), FIRST IN EQUATION %" PRId64,
                         r.numneg, r.supeqt);
            else
                snprintf(buf, sizeof buf, "PIVOT BELOW THE TOL(1) THRESHOLD IN EQUATION %" PRId64
                         " (%" PRId64 " NEGATIVE PIVOTS BEFORE IT)", r.supeqt, r.numneg);
            msg(lpu, who, buf);
        }
        c->resident = false;
    } else {
        if (r.numneg > 0) {
            ierr = 3;
            if (lpu >= 0)
                fprintf(stderr, " *** WARNING from SPR routine %s (GPU)\n     THE STIFFNESS MATRIX IS NOT POSITIVE "
                        "DEFINITE: %" PRId64 " NEGATIVE PIVOT(S)\n", who, r.numneg);
        }
        c->sm_host = sm;
        c->sm_fp = fp;
        c->resident = true;
    }
    // SPRFC4 reports SPRF41's NUMZRO there, which it never counts (sprfc4.f:258)
    mspar[25] = fc4 ? 0 : (I)r.numneg;
    return ierr;
}

// Makes the device SM hold this host SM's factor (re-uploading if needed).
// With chol the host SM is a C C' factor (SPRFC2): the device keeps its
// L D L' form, which the Cholesky solves use with a sqrt(D) scaling.
// fresh: the factorisation ran in the same call (SPRSOL with IOP <= 3), so the
// host SM cannot have changed since.
int ensure_factor_on_device(Ctx* c, const I* mspar, const double* sm, bool chol = false, bool fresh = false) {
    const int64_t nsm = mspar[7] + mspar[15];
    if (c->resident && c->sm_host == sm && c->dev_chol == chol &&
        (fresh || trust_sm() || c->sm_fp == sprb::sm_hash_host(sm, nsm, host_threads())))
        return 0;
    if (cudaMemcpyAsync(c->d_sm, sm, nsm * sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        return -4;
    uint64_t fp = 0;
    if (c->eng.hash(c->d_sm, nsm, fp) != 0) return -4;
    c->eng.invalidate_factor();
    if (chol && c->eng.chol_convert(c->d_sm, false) != 0) return -4;
    c->dev_chol = chol;
    c->sm_host = sm;
    c->sm_fp = fp;
    c->resident = true;
    return 0;
}

// Forward (which=1), back (2) or both (3) for B(LDB,NRHS) on the host; with
// chol the C C' sweeps of SPRFS2 (which=1) or SPRBS2 (which=2).
int do_solve(Ctx* c, I* mspar, I* msifa, const double* sm, double* b, I ldb, I nrhs, int which,
             bool chol = false, bool fresh = false) {
    const int64_t neq = (mspar[56] == 1 && ldb < mspar[7]) ? (int64_t)ldb : (int64_t)mspar[7];
    if (nrhs <= 0) return 0;
    if (ensure_factor_on_device(c, mspar, sm, chol, fresh) != 0) return -4;
    if (ensure_b(c, (int64_t)mspar[7] * nrhs) != 0) return -4;
    cudaStream_t s = c->stream;
    const bool peri2e = mspar[57] >= 1;                 // sprfs1.f:240-250, SPRFB3/SPRFB4
    std::vector<double> tmp;
    const int64_t nfull = mspar[7];
    if (neq != nfull && !reduced_rows_retained(c, msifa, neq, peri2e)) return -5;
    if (peri2e || neq != nfull) {
        tmp.assign(nfull * nrhs, 0.0);
        const I* p2e = msifa;                           // PERI2E = MSIFA(1..NEQ)
        for (int64_t r = 0; r < nrhs; ++r)
            for (int64_t k = 0; k < nfull; ++k) {
                const int64_t src = peri2e ? (int64_t)p2e[k] - 1 : k;
                tmp[r * nfull + k] = (src < neq) ? b[r * ldb + src] : 0.0;
            }
        if (cudaMemcpyAsync(c->d_b, tmp.data(), tmp.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
            return -4;
    } else if (ldb == nfull) {
        if (cudaMemcpyAsync(c->d_b, b, nfull * nrhs * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
            return -4;
    } else {
        if (cudaMemcpy2DAsync(c->d_b, nfull * sizeof(double), b, ldb * sizeof(double), nfull * sizeof(double), nrhs,
                              cudaMemcpyHostToDevice, s) != cudaSuccess)
            return -4;
    }
    if (neq != nfull && which == 3) {
        // the back sweep of the reference sees the equations beyond LDB as
        // zero (sprbs1.f:189), not as the forward sweep left them
        if (c->eng.solve(c->d_sm, c->d_b, nfull, nrhs, 1) != 0) return -4;
        if (peri2e) {                                   // beyond LDB in the external numbering
            if (cudaMemcpyAsync(tmp.data(), c->d_b, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess)
                return -4;
            for (int64_t r = 0; r < nrhs; ++r)
                for (int64_t k = 0; k < nfull; ++k)
                    if ((int64_t)msifa[k] - 1 >= neq) tmp[r * nfull + k] = 0.0;
            if (cudaMemcpyAsync(c->d_b, tmp.data(), tmp.size() * sizeof(double), cudaMemcpyHostToDevice, s) !=
                cudaSuccess)
                return -4;
        } else if (cudaMemset2DAsync(c->d_b + neq, nfull * sizeof(double), 0, (nfull - neq) * sizeof(double), nrhs,
                                     s) != cudaSuccess) {
            return -4;
        }
        if (c->eng.solve(c->d_sm, c->d_b, nfull, nrhs, 2) != 0) return -4;
    } else if (chol) {
        // C^-1 b = D^1/2 (D^-1 L^-1 b);  C^-T y = L^-T (D^-1/2 y)
        if (which == 2 && c->eng.scale_sqrt_d(c->d_sm, c->d_b, nfull, nrhs, true) != 0) return -4;
        if (c->eng.solve(c->d_sm, c->d_b, nfull, nrhs, which) != 0) return -4;
        if (which == 1 && c->eng.scale_sqrt_d(c->d_sm, c->d_b, nfull, nrhs, false) != 0) return -4;
    } else if (c->eng.solve(c->d_sm, c->d_b, nfull, nrhs, which) != 0) {
        return -4;
    }
    if (peri2e || neq != nfull) {
        if (cudaMemcpyAsync(tmp.data(), c->d_b, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return -4;
        if (cudaStreamSynchronize(s) != cudaSuccess) return -4;
        const I* p2e = msifa;
        for (int64_t r = 0; r < nrhs; ++r)
            for (int64_t k = 0; k < nfull; ++k) {
                const int64_t dst = peri2e ? (int64_t)p2e[k] - 1 : k;
                if (dst < neq) b[r * ldb + dst] = tmp[r * nfull + k];
            }
    } else if (ldb == nfull) {
        if (cudaMemcpyAsync(b, c->d_b, nfull * nrhs * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return -4;
    } else {
        if (cudaMemcpy2DAsync(b, ldb * sizeof(double), c->d_b, nfull * sizeof(double), nfull * sizeof(double), nrhs,
                              cudaMemcpyDeviceToHost, s) != cudaSuccess)
            return -4;
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) return -4;
    return 0;
}

// SPRFC1 (src/SPR/sprfc1.f:5) under g_mu; returns the context (null on an
// early error).  defer: see do_factor.
Ctx* fc1_locked(I* mspar, I* mtrees, I* msifa, double* sm, double* tol, const I* lpu, I* ierr, void (*mvmult)(),
                void (*mmmult)(), bool defer) {
    if (mspar[0] < 0) {                                 // sprfc1.f:140-148
        mspar[0] = -5;
        *ierr = -1;
        msg(*lpu, "SPRFC1", "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
        return nullptr;
    }
    mspar[0] = 5;
    *ierr = 0;
    if (!fc1_lengths_ok(mspar)) {
        mspar[0] = -2;
        *ierr = -2;
        msg(*lpu, "SPRFC1", "MTREES/MSIFA/SM, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
        return nullptr;
    }
    if (!callbacks_ok(mvmult, mmmult, true)) {
        mspar[0] = -5;
        *ierr = -4;
        msg(*lpu, "SPRFC1", "MVMULT/MMMULT DO NOT COMPUTE THE LDL' UPDATES OF LMVY18/LMMY18");
        return nullptr;
    }
    int err = 0;
    Ctx* c = get_ctx(mspar, mtrees, msifa, err);
    trace("context found");
    if (!c) {
        mspar[0] = -5;
        *ierr = (err == -2) ? -2 : -4;
        msg(*lpu, "SPRFC1", "COULD NOT SET UP THE GPU CONTEXT");
        return nullptr;
    }
    *ierr = do_factor(c, mspar, sm, tol, *lpu, nullptr, false, defer);
    if (*ierr < 0 && *ierr != -3) mspar[0] = -5;
    return c;
}

}  // namespace

// Element assembly into the packed LNZ of SM (and the right-hand side SV of
// prescribed values): SPRADM/SPRAD2 (src/SPR/spradm.f:818-1002) for every
// element in order.  For J = 1..NEDOF and I = 1..J with both DOFs free,
// SM(NEQ + K) += EM(I,J), K the LNZ position of (max eq, min eq); then,
// with constraint equations (MPMCEQ/MMCEQ/TTCC, nceq > 0), the weighted
// additions of the element's slave and prescribed DOFs.  EM of element e is
// em_scale[e] * em (one reference matrix) when em_scale is given, else the
// e-th NEDOF x NEDOF column-major matrix of em.  Additions happen in the
// reference's order and rounding, so SM and SV match SPRADM bit for bit.
// nsv as SPRADM's NSV: 0 = SM only, 1 = SM and SV, -1 = SV only.
// Returns 0, -2 (|nsv| > 1: the multi-load-case SV layout is not supported)
// or -3 when an element's DOF count or pattern does not match.
template <class T>
static int assemble_host(const T* mspar, const T* mtrees, const T* msifa, const T* meqn, const T* madof,
                         const T* mpmnpc, const T* mmnpc, const T* mpmceq, const T* mmceq, const double* ttcc,
                         int64_t nceq, int64_t nel, int64_t nedof, const double* em, const double* em_scale,
                         int64_t nsv, double* sm, double* sv) {
    if (nsv < -1 || nsv > 1 || nedof < 1 || nel < 0 || nceq < 0) return -2;
    if (nceq > 0 && (!mpmceq || !mmceq || !ttcc)) return -2;
    const sprb::LnzIndex<T> lx(mspar, mtrees, msifa);
    const int64_t neq = mspar[7];
    double* lnz = sm ? sm + neq : nullptr;
    std::vector<double> ems(em_scale ? (size_t)nedof * nedof : 0);
    int64_t cur = -1;
    const double* E = nullptr;
    return sprb::for_each_contribution(
        lx, meqn, madof, mpmnpc, mmnpc, mpmceq, mmceq, nceq, nel, nedof, nsv >= 0 && sm, nsv != 0 && sv,
        [&](bool to_sv, int64_t target, int64_t e, int64_t idx, int kind, int64_t jp, int64_t ip) {
            if (e != cur) {
                cur = e;
                if (em_scale) {
                    const double sc = em_scale[e];
                    for (int64_t k = 0; k < nedof * nedof; ++k) ems[k] = sc * em[k];
                    E = ems.data();
                } else {
                    E = em + e * nedof * nedof;
                }
            }
            double v;
            if (!sprb::contrib_value(kind, E[idx], ttcc, jp, ip, &v)) return;
            double& dst = to_sv ? sv[target] : lnz[target];
            dst = dst + v;
        });
}

extern "C" {

// SPRFC1 (src/SPR/sprfc1.f:5): LDL' factorisation of SM in place.
void SPR_API(sprfc1_)(I* mspar, I* mtrees, I* msifa, double* sm, double* tol, I* iwork, double* rwork, const I* lpu,
                      I* ierr, void (*mvmult)(), void (*mmmult)()) {
    (void)iwork;
    (void)rwork;
    std::lock_guard<std::mutex> lk(g_mu);
    fc1_locked(mspar, mtrees, msifa, sm, tol, lpu, ierr, mvmult, mmmult, false);
}

// SPRFC3 (src/SPR/sprfc3.f:5): LDL' factorisation that replaces singular
// pivots instead of stopping (TOL(4) scales the replacement) and reports them
// in DCOR(2,NEQ); IERR = -3 with MSPAR(27) = -(number replaced) still leaves a
// complete factor, MSPAR(1) = 5.
void SPR_API(sprfc3_)(I* mspar, I* mtrees, I* msifa, double* sm, double* tol, I* iwork, double* rwork, double* dcor,
                      const I* lpu, I* ierr, void (*mvmult)(), void (*mmmult)()) {
    (void)iwork;
    (void)rwork;
    std::lock_guard<std::mutex> lk(g_mu);
    if (mspar[0] < 0) {                                 // sprfc3.f:139-143
        mspar[0] = -5;
        *ierr = -1;
        msg(*lpu, "SPRFC3", "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
        return;
    }
    mspar[0] = 5;
    *ierr = 0;
    if (!fc1_lengths_ok(mspar)) {                       // sprfc3.f:209-234 (same checks as SPRFC1)
        mspar[0] = -2;
        *ierr = -2;
        msg(*lpu, "SPRFC3", "MTREES/MSIFA/SM, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
        return;
    }
    if (!callbacks_ok(mvmult, mmmult, true)) {
        mspar[0] = -5;
        *ierr = -4;
        msg(*lpu, "SPRFC3", "MVMULT/MMMULT DO NOT COMPUTE THE LDL' UPDATES OF LMVY18/LMMY18");
        return;
    }
    int err = 0;
    Ctx* c = get_ctx(mspar, mtrees, msifa, err);
    if (!c) {
        mspar[0] = -5;
        *ierr = (err == -2) ? -2 : -4;
        msg(*lpu, "SPRFC3", "COULD NOT SET UP THE GPU CONTEXT");
        return;
    }
    *ierr = do_factor(c, mspar, sm, tol, *lpu, dcor);
    if (*ierr == -4) mspar[0] = -5;
}

// SPRFC2 (src/SPR/sprfc2.f:5): Cholesky factorisation C C' of SM in place
// (MSPAR(1) = 6).  A non-positive pivot (d <= TOL(1)|a_jj|) stops it with
// IERR = -3 and MSPAR(27) = the equation, TOL(2) = d, TOL(3) = a_jj.
void SPR_API(sprfc2_)(I* mspar, I* mtrees, I* msifa, double* sm, double* tol, I* iwork, double* rwork, const I* lpu,
                      I* ierr, void (*mvmult)(), void (*mmmult)()) {
    (void)iwork;
    (void)rwork;
    std::lock_guard<std::mutex> lk(g_mu);
    if (mspar[0] < 0) {                                 // sprfc2.f:123-127
        mspar[0] = -6;
        *ierr = -1;
        msg(*lpu, "SPRFC2", "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
        return;
    }
    mspar[0] = 6;
    *ierr = 0;
    if (!fc1_lengths_ok(mspar)) {                       // the checks of SPRFC1
        mspar[0] = -2;
        *ierr = -2;
        msg(*lpu, "SPRFC2", "MTREES/MSIFA/SM, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
        return;
    }
    if (!callbacks_ok(mvmult, mmmult, false)) {
        mspar[0] = -6;
        *ierr = -4;
        msg(*lpu, "SPRFC2", "MVMULT/MMMULT DO NOT COMPUTE THE C C' UPDATES OF CMVY18/CMMY18");
        return;
    }
    int err = 0;
    Ctx* c = get_ctx(mspar, mtrees, msifa, err);
    if (!c) {
        mspar[0] = -6;
        *ierr = (err == -2) ? -2 : -4;
        msg(*lpu, "SPRFC2", "COULD NOT SET UP THE GPU CONTEXT");
        return;
    }
    *ierr = do_factor(c, mspar, sm, tol, *lpu, nullptr, true);
    if (*ierr == -4) mspar[0] = -6;
}

// SPRFC4 (src/SPR/sprfc4.f:5): Cholesky factorisation C C' of SM in place that
// replaces small pivots instead of stopping (SPRF47's rule, TOL(4) scales the
// replacement) and records them in DCOR(2,NEQ); a pivot below -TOL(1)|a_jj|
// stops it.  IERR = -3 with MSPAR(27) = -(number replaced) still leaves a
// complete C C' factor; MSPAR(1) = 6, MSPAR(26) = 0.
void SPR_API(sprfc4_)(I* mspar, I* mtrees, I* msifa, double* sm, double* tol, I* iwork, double* rwork, double* dcor,
                      const I* lpu, I* ierr, void (*mvmult)(), void (*mmmult)()) {
    (void)iwork;
    (void)rwork;
    std::lock_guard<std::mutex> lk(g_mu);
    if (mspar[0] < 0) {                                 // sprfc4.f:133-141
        mspar[0] = -6;
        *ierr = -1;
        msg(*lpu, "SPRFC4", "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
        return;
    }
    mspar[0] = 6;
    *ierr = 0;
    if (!fc1_lengths_ok(mspar)) {                       // sprfc4.f:203-228 (the checks of SPRFC1)
        mspar[0] = -2;
        *ierr = -2;
        msg(*lpu, "SPRFC4", "MTREES/MSIFA/SM, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
        return;
    }
    if (!callbacks_ok(mvmult, mmmult, false)) {
        mspar[0] = -6;
        *ierr = -4;
        msg(*lpu, "SPRFC4", "MVMULT/MMMULT DO NOT COMPUTE THE C C' UPDATES OF CMVY18/CMMY18");
        return;
    }
    int err = 0;
    Ctx* c = get_ctx(mspar, mtrees, msifa, err);
    if (!c) {
        mspar[0] = -6;
        *ierr = (err == -2) ? -2 : -4;
        msg(*lpu, "SPRFC4", "COULD NOT SET UP THE GPU CONTEXT");
        return;
    }
    *ierr = do_factor(c, mspar, sm, tol, *lpu, dcor, true);
    if (*ierr == -4) mspar[0] = -6;
}

// SPRFS2 / SPRBS2 (src/SPR/sprfs2.f:5, sprbs2.f:5): the forward C y = b and
// back C' x = y sweeps on a C C' factor (MSPAR(1) = 8).
static void chol_sweep(const char* who, int which, I* mspar, I* mtrees, I* msifa, double* sm, double* b,
                       const I* ldb, const I* nrhs, const I* lpu, I* ierr) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (mspar[0] < 0) {                                 // sprfs2.f:139-143, sprbs2.f:134-138
        mspar[0] = -8;
        *ierr = -1;
        msg(*lpu, who, "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
        return;
    }
    mspar[0] = 8;
    *ierr = 0;
    if (!solve_lengths_ok(mspar, *ldb)) {
        mspar[0] = -2;
        *ierr = -2;
        msg(*lpu, who, "MTREES/MSIFA/SM/B, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
        return;
    }
    int err = 0;
    Ctx* c = get_ctx(mspar, mtrees, msifa, err);
    const int rc = c ? do_solve(c, mspar, msifa, sm, b, *ldb, *nrhs, which, true) : -4;
    if (rc != 0) {
        mspar[0] = -8;
        *ierr = -4;
        solve_msg(*lpu, who, rc, "GPU CHOLESKY SOLVE FAILED");
    }
}

void SPR_API(sprfs2_)(I* mspar, I* mtrees, I* msifa, double* sm, double* b, const I* ldb, const I* nrhs, I* iwork,
                      double* rwork, const I* lpu, I* ierr) {
    (void)iwork;
    (void)rwork;
    chol_sweep("SPRFS2", 1, mspar, mtrees, msifa, sm, b, ldb, nrhs, lpu, ierr);
}

void SPR_API(sprbs2_)(I* mspar, I* mtrees, I* msifa, double* sm, double* b, const I* ldb, const I* nrhs,
                      double* rwork, const I* lpu, I* ierr) {
    (void)rwork;
    chol_sweep("SPRBS2", 2, mspar, mtrees, msifa, sm, b, ldb, nrhs, lpu, ierr);
}

// SPRFS1 (src/SPR/sprfs1.f:5): forward reduction and diagonal scaling of B.
void SPR_API(sprfs1_)(I* mspar, I* mtrees, I* msifa, double* sm, double* b, const I* ldb, const I* nrhs, I* iwork,
                      double* rwork, const I* lpu, I* ierr) {
    (void)iwork;
    (void)rwork;
    std::lock_guard<std::mutex> lk(g_mu);
    if (mspar[0] < 0) {                                 // sprfs1.f:136-144
        mspar[0] = -7;
        *ierr = -1;
        msg(*lpu, "SPRFS1", "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
        return;
    }
    mspar[0] = 7;
    *ierr = 0;
    if (!solve_lengths_ok(mspar, *ldb)) {
        mspar[0] = -2;
        *ierr = -2;
        msg(*lpu, "SPRFS1", "MTREES/MSIFA/SM/B, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
        return;
    }
    int err = 0;
    Ctx* c = get_ctx(mspar, mtrees, msifa, err);
    const int rc = c ? do_solve(c, mspar, msifa, sm, b, *ldb, *nrhs, 1) : -4;
    if (rc != 0) {
        mspar[0] = -7;
        *ierr = -4;
        solve_msg(*lpu, "SPRFS1", rc, "GPU FORWARD SOLVE FAILED");
    }
}

// SPRBS1 (src/SPR/sprbs1.f:5): back substitution of B.
void SPR_API(sprbs1_)(I* mspar, I* mtrees, I* msifa, double* sm, double* b, const I* ldb, const I* nrhs,
                      double* rwork, const I* lpu, I* ierr) {
    (void)rwork;
    std::lock_guard<std::mutex> lk(g_mu);
    if (mspar[0] < 0) {                                 // sprbs1.f:131-139
        mspar[0] = -7;
        *ierr = -1;
        msg(*lpu, "SPRBS1", "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
        return;
    }
    mspar[0] = 7;
    *ierr = 0;
    if (!solve_lengths_ok(mspar, *ldb)) {
        mspar[0] = -2;
        *ierr = -2;
        msg(*lpu, "SPRBS1", "MTREES/MSIFA/SM/B, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
        return;
    }
    int err = 0;
    Ctx* c = get_ctx(mspar, mtrees, msifa, err);
    const int rc = c ? do_solve(c, mspar, msifa, sm, b, *ldb, *nrhs, 2) : -4;
    if (rc != 0) {
        mspar[0] = -7;
        *ierr = -4;
        solve_msg(*lpu, "SPRBS1", rc, "GPU BACK SUBSTITUTION FAILED");
    }
}

// SPRSOL (src/SPR/sprsol.f:5): factor (IOP<=3), forward (2<=IOP<=5) and back
// (IOP>=3, IOP/=5) in one call.  When both sweeps run, B crosses the bus once.
void SPR_API(sprsol_)(const I* iop, I* mspar, I* mtrees, I* msifa, double* sm, double* b, const I* ldb,
                      const I* nrhs, double* tol, I* iwork, double* rwork, const I* lpu, I* ierr) {
    *ierr = 0;
    const I op = *iop;
    const bool bwd = op >= 3 && op != 5;
    std::unique_lock<std::mutex> lk(g_mu);
    trace_start();
    trace("SPRSOL entered");
    // IOP = 3: the factorisation's last downloads (pinned SM) overlap the solves
    Ctx* fc = nullptr;
    if (op <= 3) fc = fc1_locked(mspar, mtrees, msifa, sm, tol, lpu, ierr, nullptr, nullptr, op == 3);
    trace("SPRFC1 part done");
    const bool fwd = op >= 2 && op <= 5 && *ierr >= 0;
    if (fwd && bwd) {
        struct Finish {                                  // at every return below
            Ctx* c;
            ~Finish() { finish_copies(c); }
        } finish{fc};
        if (mspar[0] < 0) {
            mspar[0] = -7;
            *ierr = -1;
            msg(*lpu, "SPRFS1", "ERROR FROM PRECEDING SAM/SPR ROUTINE IS NOT CLEARED");
            return;
        }
        mspar[0] = 7;
        *ierr = 0;                                       // the solves reset IERR (sprfs1.f:143-144)
        if (!solve_lengths_ok(mspar, *ldb)) {
            mspar[0] = -2;
            *ierr = -2;
            msg(*lpu, "SPRFS1", "MTREES/MSIFA/SM/B, AND/OR IWORK/RWORK: NOT GREAT ENOUGH");
            return;
        }
        int err = 0;
        Ctx* c = get_ctx(mspar, mtrees, msifa, err);
        const int rc = c ? do_solve(c, mspar, msifa, sm, b, *ldb, *nrhs, 3, false, op <= 3) : -4;
        trace("solves done");
        const int frc = finish_copies(fc);
        trace("copies finished");
        if (rc != 0 || frc != 0) {
            mspar[0] = -7;
            *ierr = -4;
            solve_msg(*lpu, "SPRSOL", rc, "GPU SOLVE FAILED");
        }
        return;
    }
    if (finish_copies(fc) != 0 && *ierr >= 0) {
        mspar[0] = -5;
        *ierr = -4;
        msg(*lpu, "SPRSOL", "GPU COPY OF THE FACTOR FAILED");
        return;
    }
    lk.unlock();
    if (fwd) SPR_API(sprfs1_)(mspar, mtrees, msifa, sm, b, ldb, nrhs, iwork, rwork, lpu, ierr);
    if (bwd && !fwd && *ierr >= 0) SPR_API(sprbs1_)(mspar, mtrees, msifa, sm, b, ldb, nrhs, rwork, lpu, ierr);
}

// ---------------------------------------------------------------------------
// Device-level API: factor/solve on device-resident SM and B.
// ---------------------------------------------------------------------------
int SPR_API(spr_b200_open)(const I* mspar, const I* mtrees, const I* msifa, void** handle) {
    std::unique_ptr<Engine> e(new Engine());
    std::vector<int64_t> ms(60, 0);
    for (int i = 0; i < 58; ++i) ms[i] = (int64_t)mspar[i];
    std::vector<int64_t> mt = widen(mtrees, mspar[3]), mf = widen(msifa, mspar[2]);
    int rc = e->open(ms.data(), mt.data(), mf.data());
    if (rc != 0) return rc;
    *handle = e.release();
    return 0;
}

void SPR_API(spr_b200_close)(void* handle) { delete static_cast<Engine*>(handle); }

int SPR_API(spr_b200_set_stream)(void* handle, void* stream) {
    static_cast<Engine*>(handle)->set_stream((cudaStream_t)stream);
    return 0;
}

// out[0]=TOL(2) out[1]=TOL(3) out[2]=NUMNEG out[3]=SUPEQT out[4]=LIERR
int SPR_API(spr_b200_factor_dev)(void* handle, double* d_sm, double tol1, double* out) {
    FactorResult r;
    int rc = static_cast<Engine*>(handle)->factor(d_sm, tol1, r);
    if (rc != 0) return rc;
    out[0] = r.tol2;
    out[1] = r.tol3;
    out[2] = (double)r.numneg;
    out[3] = (double)r.supeqt;
    out[4] = (double)r.lierr;
    return 0;
}

// SPRFC3 semantics on device buffers: tol = {TOL(1), TOL(4)}, d_dcor = the
// device DCOR(2,NEQ); out as spr_b200_factor_dev, LIERR = -31 with
// SUPEQT = the number of replaced pivots when any was replaced.
int SPR_API(spr_b200_factor3_dev)(void* handle, double* d_sm, const double* tol, double* d_dcor, double* out) {
    FactorResult r;
    Engine::Singular fc3{tol[1], d_dcor};
    int rc = static_cast<Engine*>(handle)->factor(d_sm, tol[0], r, &fc3);
    if (rc != 0) return rc;
    out[0] = r.tol2;
    out[1] = r.tol3;
    out[2] = (double)r.numneg;
    out[3] = (double)r.supeqt;
    out[4] = (double)r.lierr;
    return 0;
}

int SPR_API(spr_b200_solve_dev)(void* handle, const double* d_sm, double* d_b, int64_t ldb, int64_t nrhs, int which) {
    return static_cast<Engine*>(handle)->solve(d_sm, d_b, ldb, nrhs, which);
}

// info[0]=RINFO(3) factor flops, [1]=RINFO(4)-style solve flops per RHS,
// [2]=front arena bytes, [3]=levels, [4]=last factor ms, [5]=last solve ms,
// [6]=kernel launches of the last factorisation, [7]=Schur-update launches,
// [8]=Schur-update ms (profile mode), [9]=Schur-update algorithmic flops,
// [10]=kernel launches of the last solve, [11]=NZEROL, [12]=pivots the
// mixed-mode inertia guard counted in the last factorisation, [13]=1 if that
// factorisation was redone in FP64 by the guard, [14]=trace of the original
// diagonal (sprfc1.f:483) of the last factorisation.
int SPR_API(spr_b200_info)(void* handle, double* info) {
    Engine* e = static_cast<Engine*>(handle);
    const sprb::Plan& p = e->plan();
    info[0] = p.factor_flops;
    info[1] = p.solve_flops;
    info[2] = (double)p.arena_doubles * 8.0;
    info[3] = (double)p.levels.size();
    info[4] = e->timing.factor_ms;
    info[5] = e->timing.solve_ms;
    info[6] = (double)e->timing.launches;
    info[7] = (double)e->timing.gemm_launches;
    info[8] = e->timing.gemm_ms;
    info[9] = p.gemm_flops;
    info[10] = (double)e->timing.solve_launches;
    info[11] = (double)p.nzerol;
    info[12] = (double)e->last_near_pivots();
    info[13] = e->last_refactored() ? 1.0 : 0.0;
    info[14] = e->last_trace();
    return 0;
}

// Per-supernode negative-pivot counts and first failing column (-1 if none)
// of the last factorisation (host arrays of NSUPER entries).
int SPR_API(spr_b200_sn_stats)(void* handle, int32_t* neg, int32_t* fail) {
    return static_cast<Engine*>(handle)->sn_stats(neg, fail);
}

// Residual operator of iterative refinement: CSR of the FP64 matrix held in
// the assembled (not yet factored) device SM.
int SPR_API(spr_b200_build_residual)(void* handle, const double* d_sm_assembled) {
    return static_cast<Engine*>(handle)->build_residual(d_sm_assembled);
}

// Iterative refinement on a factored device SM: x = solve(b), then
// x += solve(b - K x) until the normwise backward error <= tol.
// out[0] = correction steps, out[1] = backward error, out[2] = solve ms.
int SPR_API(spr_b200_refine)(void* handle, const double* d_sm, const double* d_b, double* d_x, int64_t ld,
                             int64_t nrhs, double tol, int maxit, double* out) {
    return static_cast<Engine*>(handle)->refine(d_sm, d_b, d_x, ld, nrhs, tol, maxit, out);
}

// Factorisation mode: 0 = FP64 (the drop-in), 1 = mixed (3xTF32 Schur updates).
int SPR_API(spr_b200_set_mode)(void* handle, int mode) {
    if (mode < 0 || mode > 2) return -2;
    static_cast<Engine*>(handle)->set_mixed(mode);
    return 0;
}

// Split across GPUs: node mask (NSUPER bytes, nonzero = another rank's; null
// clears it) and the exchange lists of the following factorisations
// (update blocks) and forward sweeps (update vectors).
int SPR_API(spr_b200_set_skip)(void* handle, const uint8_t* mask) {
    return static_cast<Engine*>(handle)->set_skip(mask);
}

int SPR_API(spr_b200_set_exchange)(void* handle, int64_t nfo, const int32_t* fo_node, double* const* fo_buf,
                                   int64_t nfi, const int32_t* fi_node, double* const* fi_buf, int64_t nvo,
                                   const int32_t* vo_node, double* const* vo_buf, int64_t nvi, const int32_t* vi_node,
                                   double* const* vi_buf) {
    Engine* e = static_cast<Engine*>(handle);
    const int64_t ns = e->plan().nsuper;
    auto list = [ns](int64_t n, const int32_t* node, double* const* buf, std::vector<Engine::Xfer>& out) {
        out.clear();
        for (int64_t k = 0; k < n; ++k) {
            if (node[k] < 0 || node[k] >= ns || !buf[k]) return false;
            out.push_back(Engine::Xfer{node[k], buf[k]});
        }
        return true;
    };
    std::vector<Engine::Xfer> fo, fi, vo, vi;
    if (!list(nfo, fo_node, fo_buf, fo) || !list(nfi, fi_node, fi_buf, fi) || !list(nvo, vo_node, vo_buf, vo) ||
        !list(nvi, vi_node, vi_buf, vi))
        return -2;
    e->set_exchange(std::move(fo), std::move(fi), std::move(vo), std::move(vi));
    return 0;
}

// Inertia guard of the mixed mode (default tau = 1e-3; 0 = off).
int SPR_API(spr_b200_set_inertia_guard)(void* handle, double tau) {
    if (!(tau >= 0.0)) return -2;
    static_cast<Engine*>(handle)->set_inertia_guard(tau);
    return 0;
}

// Watchdog of the tensor-core update: wait limit (ns, > 0) and the test
// switch that makes one CTA's waits run out.
int SPR_API(spr_b200_set_watchdog)(void* handle, double wait_ns, int drop) {
    if (!(wait_ns >= 1.0e6 && wait_ns <= 6.0e10)) return -2;
    static_cast<Engine*>(handle)->set_watchdog((unsigned long long)wait_ns, drop != 0);
    return 0;
}

// Profile mode: CUDA events around every Schur-update launch (spr_b200_info[8]).
// Profile mode only: factor time of the last factorisation by phase
// (out[0..8]: pre-pass, small fronts, extend-add, diagonal blocks, panel
// TRSM, in-panel/trailing updates, K = S update, write-back, end) and of the
// last solve (out[9..19], see Timing::phase_ms).
int SPR_API(spr_b200_phase_ms)(void* handle, double* out) {
    const auto& t = static_cast<Engine*>(handle)->timing;
    for (int k = 0; k < 20; ++k) out[k] = t.phase_ms[k];
    return 0;
}

// Mixed-mode autotuner: which Schur updates run on the tensor cores and how
// many SMs the side-stream launches take, timed on a copy of the assembled SM.
int SPR_API(spr_b200_autotune)(void* handle, const double* d_sm_assembled, double* out) {
    return static_cast<Engine*>(handle)->autotune(d_sm_assembled, out);
}

// Self-test of the pivot reciprocal (host arrays): out[2i] = the device's
// reciprocal of x[i], out[2i+1] = the IEEE quotient 1.0 / x[i].
int SPR_API(spr_b200_recip_check)(const double* x, int64_t n, double* out) { return sprb::recip_check(x, n, out); }

// Tile autotuner of the small FP64 Schur updates (see Engine::autotune_tiles):
// out[0] = tile chosen (64 or 32), out[1] / out[2] = factor ms with each.
int SPR_API(spr_b200_autotune_tiles)(void* handle, const double* d_sm_assembled, double* out) {
    return static_cast<Engine*>(handle)->autotune_tiles(d_sm_assembled, out);
}

// Sets the tile of the small FP64 Schur updates (64 or 32).
int SPR_API(spr_b200_set_small_tile)(void* handle, int tile) {
    static_cast<Engine*>(handle)->set_small_tile(tile);
    return 0;
}

// Mixed mode: out[0] = algorithmic flops of the updates that ran on tensor
// cores in the last profiled factorisation (far trailing columns, the next
// super-panels' columns and K = S updates above the tensor-core
// threshold), out[1] = their split + tensor-core time (ms).
int SPR_API(spr_b200_tc_stats)(void* handle, double* out) {
    const Engine* e = static_cast<Engine*>(handle);
    out[0] = e->timing.tc_flops;
    out[1] = e->timing.tc_ms;
    return 0;
}

int SPR_API(spr_b200_set_profile)(void* handle, int on) {
    static_cast<Engine*>(handle)->set_profile(on != 0);
    return 0;
}

// Host-only: builds the plan and self-checks it (no GPU needed).
// out[0]=rc [1]=NSUPER [2]=levels [3]=arena doubles [4]=buffers out of bounds
// [5]=overlapping live buffers [6]=factor flops (RINFO(3)) [7]=solve flops
// [8]=small fronts [9]=large fronts [10]=jobs
int SPR_API(spr_b200_plan_check)(const I* mspar, const I* mtrees, const I* msifa, double* out) {
    std::vector<int64_t> ms(60, 0);
    for (int i = 0; i < 58; ++i) ms[i] = (int64_t)mspar[i];
    std::vector<int64_t> mt = widen(mtrees, mspar[3]), mf = widen(msifa, mspar[2]);
    sprb::Plan p;
    const int rc = sprb::build_plan(ms.data(), mt.data(), mf.data(), p);
    for (int i = 0; i < 13; ++i) out[i] = 0.0;
    out[0] = rc;
    if (rc != 0) return rc;
    int64_t oob = 0, ov = 0;
    sprb::check_plan(p, oob, ov);
    int64_t nsmall = 0, nlarge = 0;
    for (const auto& lp : p.levels) {
        nsmall += (int64_t)lp.small_nodes.size();
        nlarge += (int64_t)lp.large_nodes.size();
    }
    out[1] = (double)p.nsuper;
    out[2] = (double)p.levels.size();
    out[3] = (double)p.arena_doubles;
    out[4] = (double)oob;
    out[5] = (double)ov;
    out[6] = p.factor_flops;
    out[7] = p.solve_flops;
    out[8] = (double)nsmall;
    out[9] = (double)nlarge;
    out[10] = (double)p.jobs.size();
    int64_t cf = 0, ct = 0;
    sprb::check_coverage(p, cf, ct);
    out[11] = (double)cf;
    out[12] = (double)ct;
    return 0;
}

// Host-only race check of the factorisation's stream schedule (no GPU needed):
// out[0] = ordering violations of the FP64 schedule, out[1] = of the schedule
// with tensor-core far and K = S updates, out[2] = of the FP64 schedule without
// its side-stream joins (a self-test of the check), out[3] = far launches,
// out[4] = violations without the look-ahead joins, out[5] = look-ahead launches.
int SPR_API(spr_b200_schedule_check)(const I* mspar, const I* mtrees, const I* msifa, double* out) {
    std::vector<int64_t> ms(60, 0);
    for (int i = 0; i < 58; ++i) ms[i] = (int64_t)mspar[i];
    std::vector<int64_t> mt = widen(mtrees, mspar[3]), mf = widen(msifa, mspar[2]);
    sprb::Plan p;
    const int rc = sprb::build_plan(ms.data(), mt.data(), mf.data(), p);
    for (int i = 0; i < 6; ++i) out[i] = 0.0;
    if (rc != 0) return rc;
    out[0] = (double)sprb::check_schedule(p, false, 0);
    out[1] = (double)sprb::check_schedule(p, true, 0);
    out[2] = (double)sprb::check_schedule(p, false, 1);
    out[4] = (double)sprb::check_schedule(p, false, 2);
    int64_t nfar = 0, nahead = 0;
    for (const auto& lp : p.levels) {
        for (const auto& v : lp.far) nfar += (int64_t)v.size();
        for (const auto& v : lp.ahead) nahead += (int64_t)v.size();
    }
    out[3] = (double)nfar;
    out[5] = (double)nahead;
    return 0;
}

// Host-only check of the solves' plan (no GPU needed): out[0] = rc,
// out[1] = violations of the plan as built, out[2] = triangle tasks checked,
// out[3] and out[4] = violations reported with a planted mistake (two blocks
// of a front swapped; one front's forward partials moved onto another's),
// -1 where the structure has no front the mistake applies to.
int SPR_API(spr_b200_solve_plan_check)(const I* mspar, const I* mtrees, const I* msifa, double* out) {
    std::vector<int64_t> ms(60, 0);
    for (int i = 0; i < 58; ++i) ms[i] = (int64_t)mspar[i];
    std::vector<int64_t> mt = widen(mtrees, mspar[3]), mf = widen(msifa, mspar[2]);
    sprb::Plan p;
    const int rc = sprb::build_plan(ms.data(), mt.data(), mf.data(), p);
    for (int i = 0; i < 5; ++i) out[i] = 0.0;
    out[0] = rc;
    if (rc != 0) return rc;
    int64_t ntask = 0;
    out[1] = (double)sprb::check_solve_plan(p, 0, &ntask);
    out[2] = (double)ntask;
    out[3] = (double)sprb::check_solve_plan(p, 1);
    out[4] = (double)sprb::check_solve_plan(p, 2);
    return 0;
}

// Host SPRADM restatements; see assemble_host.
int SPR_API(spr_b200_assemble)(const I* mspar, const I* mtrees, const I* msifa, const I* meqn, const I* madof,
                               const I* mpmnpc, const I* mmnpc, I nel, I nedof, const double* em,
                               const double* em_scale, double* sm) {
    return assemble_host<I>(mspar, mtrees, msifa, meqn, madof, mpmnpc, mmnpc, nullptr, nullptr, nullptr, 0, nel,
                            nedof, em, em_scale, 0, sm, nullptr);
}

int SPR_API(spr_b200_assemble_ceq)(const I* mspar, const I* mtrees, const I* msifa, const I* meqn,
                                   const I* madof, const I* mpmnpc, const I* mmnpc, const I* mpmceq,
                                   const I* mmceq, const double* ttcc, I nceq, I nel, I nedof, const double* em,
                                   const double* em_scale, I nsv, double* sm, double* sv) {
    return assemble_host<I>(mspar, mtrees, msifa, meqn, madof, mpmnpc, mmnpc, mpmceq, mmceq, ttcc, nceq, nel,
                            nedof, em, em_scale, nsv, sm, sv);
}

// Element-level device operations (assembly gather, hex8 stiffness, adjoint
// element gradient) on one structure and one SAM element topology.
static int elem_open(const I* mspar, const I* mtrees, const I* msifa, const I* meqn, const I* madof,
                     const I* mpmnpc, const I* mmnpc, const I* mpmceq, const I* mmceq, I nceq, I nel, I nedof,
                     void** handle) {
    if (nel < 0 || nceq < 0) return -2;
    std::vector<int64_t> ms(60, 0);
    for (int i = 0; i < 58; ++i) ms[i] = (int64_t)mspar[i];
    std::vector<int64_t> mt = widen(mtrees, mspar[3]), mf = widen(msifa, mspar[2]);
    std::vector<int64_t> pn = widen(mpmnpc, nel + 1);
    std::vector<int64_t> mn = widen(mmnpc, pn[nel] - 1);
    int64_t nnod = 0;
    for (int64_t v : mn) nnod = std::max(nnod, v);
    std::vector<int64_t> pc = nceq > 0 ? widen(mpmceq, nceq + 1) : std::vector<int64_t>();
    std::vector<int64_t> mc = nceq > 0 ? widen(mmceq, pc[nceq] - 1) : std::vector<int64_t>();
    std::vector<int64_t> ad = widen(madof, nnod + 1);
    int64_t ndof = nnod > 0 ? ad[nnod] - 1 : 0;
    for (int64_t v : mc) ndof = std::max(ndof, v);      // MMCEQ holds DOF numbers
    std::vector<int64_t> eq = widen(meqn, ndof);
    std::unique_ptr<sprb::Elements> e(new sprb::Elements());
    const int rc = e->open(ms.data(), mt.data(), mf.data(), eq.data(), ad.data(), pn.data(), mn.data(), nel, nedof,
                           nceq > 0 ? pc.data() : nullptr, nceq > 0 ? mc.data() : nullptr, nceq);
    if (rc != 0) return rc;
    *handle = e.release();
    return 0;
}

int SPR_API(spr_b200_elem_open)(const I* mspar, const I* mtrees, const I* msifa, const I* meqn, const I* madof,
                                const I* mpmnpc, const I* mmnpc, I nel, I nedof, void** handle) {
    return elem_open(mspar, mtrees, msifa, meqn, madof, mpmnpc, mmnpc, nullptr, nullptr, 0, nel, nedof, handle);
}

int SPR_API(spr_b200_elem_open_ceq)(const I* mspar, const I* mtrees, const I* msifa, const I* meqn,
                                    const I* madof, const I* mpmnpc, const I* mmnpc, const I* mpmceq,
                                    const I* mmceq, I nceq, I nel, I nedof, void** handle) {
    return elem_open(mspar, mtrees, msifa, meqn, madof, mpmnpc, mmnpc, mpmceq, mmceq, nceq, nel, nedof, handle);
}

void SPR_API(spr_b200_elem_close)(void* handle) { delete static_cast<sprb::Elements*>(handle); }

int SPR_API(spr_b200_elem_assemble)(void* handle, double* d_sm, const double* d_em, const double* d_scale,
                                    void* stream) {
    return static_cast<sprb::Elements*>(handle)->assemble(d_sm, d_em, d_scale, (cudaStream_t)stream);
}

int SPR_API(spr_b200_elem_assemble_ceq)(void* handle, double* d_sm, double* d_sv, const double* d_em,
                                        const double* d_scale, const double* d_ttcc, void* stream) {
    return static_cast<sprb::Elements*>(handle)->assemble(d_sm, d_em, d_scale, (cudaStream_t)stream, d_sv, d_ttcc);
}

int SPR_API(spr_b200_elem_hex8)(void* handle, const double* d_xyz, const double* d_E, double nu, double* d_em,
                                void* stream) {
    return static_cast<sprb::Elements*>(handle)->hex8(d_xyz, d_E, nu, d_em, (cudaStream_t)stream);
}

int SPR_API(spr_b200_elem_grad)(void* handle, const double* d_u, const double* d_lam, int64_t ld, int64_t nrhs,
                                const double* d_em, const double* d_dscale, double* d_grad, void* stream) {
    return static_cast<sprb::Elements*>(handle)->grad(d_u, d_lam, ld, nrhs, d_em, d_dscale, d_grad,
                                                      (cudaStream_t)stream);
}

// Releases every cached context (device memory of the Fortran entry points).
// Timing of the last factorisation through the Fortran entry points with a
// pinned SM: out[0] = ms of upload before the factorisation could start,
// out[1] = factorisation ms, out[2] = ms of download after it.
int SPR_API(spr_b200_copy_stats)(double* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (int k = 0; k < 3; ++k) out[k] = g_copy_ms[k];
    return 0;
}

// Number of device contexts the Fortran entry points hold (one per
// structure triple they were called with); 0 before any call.
int SPR_API(spr_b200_contexts)(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    return (int)g_ctx.size();
}

void SPR_API(spr_b200_release_all)(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_ctx.clear();
}

}  // extern "C"
