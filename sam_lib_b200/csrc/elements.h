// Element-level device operations on one SPR structure: assembly of SM (and
// of the prescribed-value right-hand side SV) from element matrices (SPRAD2,
// src/SPR/spradm.f:741-1005, as a deterministic gather), the hex8 element
// stiffness from nodal coordinates, and the adjoint element gradient
// g_e = -sum_q lambda_q,e^T (dK_e/dtheta_e) u_q,e.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace sprb {

// How one SPRAD2 addition weights its element-matrix entry EM(I,J); t = TTCC.
enum ContribKind : uint8_t {
    kFree = 0,           // SM(K) + EM(I,J)                               (spradm.f:856)
    kMaster = 1,         // SM(K) + t(JP)*EM(I,J), I free, J a slave      (:949)
    kMasterDiag = 2,     // SM(K) + (t(JP)+t(JP))*EM(I,J), I the master   (:966)
    kMasterMaster = 3,   // SM(K) + t(IP)*t(JP)*EM(I,J), both slaves      (:997)
    kSvFree = 4,         // SV(K) - C0*EM(I,J), C0 = t(MPMCEQ(JCEQ))       (:893)
    kSvMaster = 5,       // SV(K) - C0*t(IP)*EM(I,J), I a slave            (:904)
};

// LNZ position of entry (row, col), row >= col, of the packed supernodal
// lower triangle (column j of supernode JS at XLNZ(JS) + j*F - j(j-1)/2,
// rows in LINDX order), or -1 outside the symbolic pattern.  0-based result
// from the 1-based SPR arrays.
template <class T>
struct LnzIndex {
    const T *xsuper, *xlindx, *lindx, *xlnz;
    std::vector<int32_t> colsn;
    LnzIndex(const T* mspar, const T* mtrees, const T* msifa)
        : xsuper(mtrees + (mspar[44] - 1)), xlindx(mtrees + (mspar[45] - 1)), lindx(msifa + (mspar[46] - 1)),
          xlnz(msifa + (mspar[47] - 1)), colsn(mspar[7]) {
        for (int64_t js = 0; js < mspar[10]; ++js)
            for (int64_t c = xsuper[js]; c < xsuper[js + 1]; ++c) colsn[c - 1] = (int32_t)js;
    }
    int64_t pos(int64_t row, int64_t col) const {
        const int64_t js = colsn[col - 1];
        const int64_t F = xlindx[js + 1] - xlindx[js];
        const T* rows = lindx + (xlindx[js] - 1);
        int64_t lo = col - xsuper[js], hi = F - 1;      // the row is at or below the column
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((int64_t)rows[mid] < row) lo = mid + 1;
            else hi = mid;
        }
        if ((int64_t)rows[lo] != row) return -1;
        const int64_t jc = col - xsuper[js];
        return (xlnz[js] - 1) + jc * F - (jc * (jc - 1)) / 2 + (lo - jc);
    }
};

__host__ __device__ inline double rn_mul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}

__host__ __device__ inline double rn_add(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}

// The value SPRAD2 adds for one contribution of kind `kind` on the element
// entry em, rounded as the reference evaluates it (left to right, one
// rounding per operation; a subtraction adds the negated product, which is
// the same number).  Returns false where a zero TTCC coefficient or C0 makes
// SPRAD2 skip the addition (spradm.f:874, :902, :917, :979).
__host__ __device__ inline bool contrib_value(int kind, double em, const double* ttcc, int64_t jp, int64_t ip,
                                              double* v) {
    switch (kind) {
        case kFree:
            *v = em;
            return true;
        case kMaster:
        case kMasterDiag: {
            const double t = ttcc[jp - 1];
            if (t == 0.0) return false;
            *v = rn_mul(kind == kMaster ? t : rn_add(t, t), em);
            return true;
        }
        case kMasterMaster: {
            const double tj = ttcc[jp - 1], ti = ttcc[ip - 1];
            if (tj == 0.0 || ti == 0.0) return false;
            *v = rn_mul(rn_mul(ti, tj), em);
            return true;
        }
        case kSvFree: {
            const double c0 = ttcc[jp - 1];
            if (c0 == 0.0) return false;
            *v = -rn_mul(c0, em);
            return true;
        }
        case kSvMaster: {
            const double c0 = ttcc[jp - 1], ti = ttcc[ip - 1];
            if (c0 == 0.0 || ti == 0.0) return false;
            *v = -rn_mul(rn_mul(c0, ti), em);
            return true;
        }
    }
    return false;
}

// Visits the additions SPRADM makes for every element, in its order
// (elements in order; per element SPRAD2's free-DOF loop J = 1..NEDOF,
// I = 1..J, src/SPR/spradm.f:818-859, then per constrained DOF J its SV part
// and its master loop, :868-1002), calling
//     f(to_sv, target, e, I + J*nedof, kind, jp, ip)
// with target the 0-based LNZ position (to_sv false) or SV index (true) and
// jp/ip 1-based positions in MMCEQ/TTCC.  Value tests on TTCC (a zero
// coefficient or C0 skips the addition) are left to the caller, who has the
// values.  want_sm/want_sv follow NSV: 0 -> SM only, 1 -> both, -1 -> SV
// only.  Topology arrays are SAM's, 1-based contents; nceq = 0 when the
// system has no constraint equations (mpmceq/mmceq are then not read).
// Returns 0, or -3 on a DOF count or pattern mismatch.
template <class T, class F>
int for_each_contribution(const LnzIndex<T>& lx, const T* meqn, const T* madof, const T* mpmnpc, const T* mmnpc,
                          const T* mpmceq, const T* mmceq, int64_t nceq, int64_t nel, int64_t nedof, bool want_sm,
                          bool want_sv, F&& f) {
    std::vector<int64_t> meen(nedof);
    for (int64_t e = 0; e < nel; ++e) {
        int64_t nd = 0, nceq_e = 0;
        for (int64_t p = mpmnpc[e]; p < (int64_t)mpmnpc[e + 1]; ++p) {
            const int64_t node = mmnpc[p - 1];
            for (int64_t d = madof[node - 1]; d < (int64_t)madof[node]; ++d) {
                if (nd >= nedof) return -3;
                meen[nd] = (int64_t)meqn[d - 1];
                if (meen[nd] < 0) ++nceq_e;
                ++nd;
            }
        }
        if (nd != nedof) return -3;
        if (want_sm) {
            for (int64_t J = 0; J < nedof; ++J) {
                const int64_t jeq = meen[J];
                if (jeq < 1) continue;
                for (int64_t Iq = 0; Iq <= J; ++Iq) {
                    const int64_t ieq = meen[Iq];
                    if (ieq < 1) continue;
                    const int64_t k = lx.pos(std::max(ieq, jeq), std::min(ieq, jeq));
                    if (k < 0) return -3;
                    f(false, k, e, Iq + J * nedof, kFree, int64_t(0), int64_t(0));
                }
            }
        }
        if (nceq == 0 || nceq_e == 0) continue;
        for (int64_t J = 0; J < nedof; ++J) {
            if (meen[J] >= 0) continue;
            const int64_t jceq = -meen[J];
            if (jceq > nceq) return -3;
            const int64_t jp0 = (int64_t)mpmceq[jceq - 1];
            const int64_t idx = J * nedof;
            if (want_sv) {
                for (int64_t Iq = 0; Iq < nedof; ++Iq) {
                    const int64_t ieq = meen[Iq];
                    if (ieq == 0) continue;
                    if (ieq > 0) {
                        f(true, ieq - 1, e, Iq + idx, kSvFree, jp0, int64_t(0));
                        continue;
                    }
                    const int64_t iceq = -ieq;
                    for (int64_t ip = (int64_t)mpmceq[iceq - 1] + 1; ip < (int64_t)mpmceq[iceq]; ++ip) {
                        if (mmceq[ip - 1] <= 0) continue;
                        f(true, (int64_t)meqn[mmceq[ip - 1] - 1] - 1, e, Iq + idx, kSvMaster, jp0, ip);
                    }
                }
            }
            if (!want_sm) continue;
            for (int64_t jp = jp0 + 1; jp < (int64_t)mpmceq[jceq]; ++jp) {
                if (mmceq[jp - 1] <= 0) continue;
                const int64_t jeq = (int64_t)meqn[mmceq[jp - 1] - 1];
                for (int64_t Iq = 0; Iq < nedof; ++Iq) {
                    const int64_t ieq = meen[Iq];
                    if (ieq == 0) continue;
                    if (ieq > 0) {
                        const int64_t k = lx.pos(std::max(ieq, jeq), std::min(ieq, jeq));
                        if (k < 0) return -3;
                        f(false, k, e, Iq + idx, ieq != jeq ? kMaster : kMasterDiag, jp, int64_t(0));
                        continue;
                    }
                    const int64_t iceq = -ieq;
                    for (int64_t ip = (int64_t)mpmceq[iceq - 1] + 1; ip < (int64_t)mpmceq[iceq]; ++ip) {
                        if (mmceq[ip - 1] <= 0) continue;
                        const int64_t ieq2 = (int64_t)meqn[mmceq[ip - 1] - 1];
                        if (ieq2 > jeq) continue;
                        const int64_t k = lx.pos(jeq, ieq2);
                        if (k < 0) return -3;
                        f(false, k, e, Iq + idx, kMasterMaster, jp, ip);
                    }
                }
            }
        }
    }
    return 0;
}

class Elements {
public:
    ~Elements();
    // Host build from the structure (MSPAR/MTREES/MSIFA) and the SAM element
    // topology (MEQN, MADOF, MPMNPC, MMNPC; 1-based as in SAM), with the
    // constraint equations MPMCEQ/MMCEQ (nceq of them; nceq = 0 and null
    // pointers without).  Every element must have exactly nedof DOFs.
    // Returns 0, -2 (nedof > 32 or nel >= 2^22) or -3 (DOF count or pattern
    // mismatch), -4 on CUDA errors.
    int open(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa, const int64_t* meqn,
             const int64_t* madof, const int64_t* mpmnpc, const int64_t* mmnpc, int64_t nel, int64_t nedof,
             const int64_t* mpmceq = nullptr, const int64_t* mmceq = nullptr, int64_t nceq = 0);
    // SM = 0, then LNZ(k) = sum over contributing (e, I, J) in element order of
    // EM_e(I,J); EM_e = scale[e] * em when scale is given, else em + e*nedof^2.
    // The sum runs in SPRADM's order with separately rounded products, so
    // the result equals the host assembly bit for bit.  With constraint
    // equations the weighted additions of SPRAD2 take part (TTCC on the
    // device, d_ttcc), and d_sv (NEQ, zeroed first) receives the prescribed
    // values' right-hand side; d_sm or d_sv may be null (NSV = -1 or 0).
    int assemble(double* d_sm, const double* d_em, const double* d_scale, cudaStream_t s,
                 double* d_sv = nullptr, const double* d_ttcc = nullptr);
    // em + e*576 = the 24x24 stiffness (node-major DOFs, column-major) of the
    // hex8 element e from the node coordinates xyz (NANOD x 3, by SAM node
    // number - 1), isoparametric with 2x2x2 Gauss, isotropic with Young's
    // modulus E[e] and Poisson's ratio nu.  Returns -2 unless every element
    // has 8 nodes of 3 DOFs.
    int hex8(const double* d_xyz, const double* d_E, double nu, double* d_em, cudaStream_t s);
    // grad[e] = -sum_q lam_q(eq_e)^T dK_e u_q(eq_e), dK_e = dscale[e] * em when
    // dscale is given, else em + e*nedof^2 (column-major, full matrices).
    // u, lam: ld x nrhs, equation order.
    int grad(const double* d_u, const double* d_lam, int64_t ld, int64_t nrhs, const double* d_em,
             const double* d_dscale, double* d_grad, cudaStream_t s);
    int64_t nel() const { return nel_; }
    int64_t neq() const { return neq_; }
    int64_t contributions() const { return ncontrib_; }
    int64_t positions() const { return npos_; }

    int64_t sv_positions() const { return sv_.npos; }

private:
    // One gather plan: per target (LNZ position or SV index) its
    // contributions in the reference's order.
    struct Gather {
        int64_t npos = 0, ncontrib = 0;
        int64_t* pos = nullptr;      // targets with at least one contribution
        int64_t* cptr = nullptr;     // contributions of pos[i]: [cptr[i], cptr[i+1])
        uint32_t* contrib = nullptr; // (element << 10) | (I + J*nedof)
        uint8_t* kind = nullptr;     // ContribKind, null when every one is kFree
        int32_t* jp = nullptr;       // 1-based MMCEQ/TTCC positions (with kind)
        int32_t* ip = nullptr;
        void release();
    };
    int upload(Gather& g, std::vector<std::pair<int64_t, uint64_t>>& pc, const std::vector<int32_t>& jp,
               const std::vector<int32_t>& ip, const std::vector<uint8_t>& kind, bool weighted);
    int64_t nel_ = 0, nedof_ = 0, neq_ = 0, nzerol_ = 0, npos_ = 0, ncontrib_ = 0;
    Gather sm_, sv_;
    int32_t* eq_ = nullptr;          // nel x nedof equation numbers (0-based, -1 constrained)
    int32_t* enodes_ = nullptr;      // nel x 8 node indices (0-based) when every element is a hex8
};

}  // namespace sprb
