// Element-level device operations on one SPR structure: assembly of SM from
// element matrices (the SPRADM main add, src/SPR/spradm.f:818-859, as a
// deterministic gather) and the adjoint element gradient
// g_e = -sum_q lambda_q,e^T (dK_e/dtheta_e) u_q,e.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace sprb {

class Elements {
public:
    ~Elements();
    // Host build from the structure (MSPAR/MTREES/MSIFA) and the SAM element
    // topology (MEQN, MADOF, MPMNPC, MMNPC; 1-based as in SAM).  Every
    // element must have exactly nedof DOFs.  Returns 0, -2 (nedof > 32 or
    // nel >= 2^22) or -3 (DOF count mismatch), -4 on CUDA errors.
    int open(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa, const int64_t* meqn,
             const int64_t* madof, const int64_t* mpmnpc, const int64_t* mmnpc, int64_t nel, int64_t nedof);
    // SM = 0, then LNZ(k) = sum over contributing (e, I, J) in element order of
    // EM_e(I,J); EM_e = scale[e] * em when scale is given, else em + e*nedof^2.
    // The sum runs in SPRADM's order with separately rounded products, so
    // the result equals the host assembly bit for bit.
    int assemble(double* d_sm, const double* d_em, const double* d_scale, cudaStream_t s);
    // grad[e] = -sum_q lam_q(eq_e)^T dK_e u_q(eq_e), dK_e = dscale[e] * em when
    // dscale is given, else em + e*nedof^2 (column-major, full matrices).
    // u, lam: ld x nrhs, equation order.
    int grad(const double* d_u, const double* d_lam, int64_t ld, int64_t nrhs, const double* d_em,
             const double* d_dscale, double* d_grad, cudaStream_t s);
    int64_t nel() const { return nel_; }
    int64_t neq() const { return neq_; }
    int64_t contributions() const { return ncontrib_; }
    int64_t positions() const { return npos_; }

private:
    int64_t nel_ = 0, nedof_ = 0, neq_ = 0, nzerol_ = 0, npos_ = 0, ncontrib_ = 0;
    int64_t* pos_ = nullptr;         // LNZ positions with at least one contribution
    int64_t* cptr_ = nullptr;        // contributions of pos_[i]: [cptr_[i], cptr_[i+1])
    uint32_t* contrib_ = nullptr;    // (element << 10) | (I + J*nedof), element order
    int32_t* eq_ = nullptr;          // nel x nedof equation numbers (0-based, -1 constrained)
};

}  // namespace sprb
