// Element assembly and adjoint element gradient on the device.
#include "elements.h"

#include <algorithm>
#include <vector>

namespace sprb {

#define ECK(x)                                \
    do {                                      \
        if ((x) != cudaSuccess) return -4;    \
    } while (0)

Elements::~Elements() {
    cudaFree(pos_);
    cudaFree(cptr_);
    cudaFree(contrib_);
    cudaFree(eq_);
}

int Elements::open(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa, const int64_t* meqn,
                   const int64_t* madof, const int64_t* mpmnpc, const int64_t* mmnpc, int64_t nel,
                   int64_t nedof) {
    if (nedof < 1 || nedof > 32 || nel < 0 || nel >= (int64_t(1) << 22)) return -2;
    neq_ = mspar[7];
    nzerol_ = mspar[15];
    nel_ = nel;
    nedof_ = nedof;
    const int64_t nsuper = mspar[10];
    const int64_t* xsuper = mtrees + (mspar[44] - 1);
    const int64_t* xlindx = mtrees + (mspar[45] - 1);
    const int64_t* lindx = msifa + (mspar[46] - 1);
    const int64_t* xlnz = msifa + (mspar[47] - 1);
    std::vector<int32_t> colsn(neq_);
    for (int64_t js = 0; js < nsuper; ++js)
        for (int64_t c = xsuper[js]; c < xsuper[js + 1]; ++c) colsn[c - 1] = (int32_t)js;
    // (LNZ position, packed contribution) in SPRADM's loop order: elements in
    // order, J = 1..NEDOF, I = 1..J (spradm.f:818-859)
    std::vector<int32_t> eq((size_t)nel * nedof);
    std::vector<std::pair<int64_t, uint32_t>> pc;
    pc.reserve((size_t)nel * nedof * (nedof + 1) / 2);
    for (int64_t e = 0; e < nel; ++e) {
        int64_t nd = 0;
        for (int64_t p = mpmnpc[e]; p < mpmnpc[e + 1]; ++p) {
            const int64_t node = mmnpc[p - 1];
            for (int64_t d = madof[node - 1]; d < madof[node]; ++d) {
                if (nd >= nedof) return -3;
                const int64_t q = meqn[d - 1];
                eq[e * nedof + nd++] = q >= 1 ? (int32_t)(q - 1) : -1;
            }
        }
        if (nd != nedof) return -3;
        const int32_t* ee = eq.data() + e * nedof;
        for (int64_t J = 0; J < nedof; ++J) {
            if (ee[J] < 0) continue;
            for (int64_t I = 0; I <= J; ++I) {
                if (ee[I] < 0) continue;
                const int64_t ieq = ee[I] + 1, jeq = ee[J] + 1;
                const int64_t col = std::min(ieq, jeq), row = std::max(ieq, jeq);
                const int64_t js = colsn[col - 1];
                const int64_t F = xlindx[js + 1] - xlindx[js];
                const int64_t* rows = lindx + (xlindx[js] - 1);
                int64_t lo = col - xsuper[js], hi = F - 1;
                while (lo < hi) {
                    const int64_t mid = (lo + hi) >> 1;
                    if (rows[mid] < row) lo = mid + 1;
                    else hi = mid;
                }
                if (rows[lo] != row) return -3;      // (row, col) outside the symbolic pattern
                const int64_t jc = col - xsuper[js];
                const int64_t k = (xlnz[js] - 1) + jc * F - (jc * (jc - 1)) / 2 + (lo - jc);
                pc.emplace_back(k, (uint32_t)((e << 10) | (I + J * nedof)));
            }
        }
    }
    // group by position, keeping the element order inside each group
    std::stable_sort(pc.begin(), pc.end(),
                     [](const std::pair<int64_t, uint32_t>& a, const std::pair<int64_t, uint32_t>& b) {
                         return a.first < b.first;
                     });
    std::vector<int64_t> pos, cptr;
    std::vector<uint32_t> contrib(pc.size());
    for (size_t i = 0; i < pc.size(); ++i) {
        if (i == 0 || pc[i].first != pc[i - 1].first) {
            pos.push_back(pc[i].first);
            cptr.push_back((int64_t)i);
        }
        contrib[i] = pc[i].second;
    }
    cptr.push_back((int64_t)pc.size());
    npos_ = (int64_t)pos.size();
    ncontrib_ = (int64_t)pc.size();
    ECK(cudaMalloc((void**)&pos_, std::max<int64_t>(npos_, 1) * sizeof(int64_t)));
    ECK(cudaMalloc((void**)&cptr_, (npos_ + 1) * sizeof(int64_t)));
    ECK(cudaMalloc((void**)&contrib_, std::max<int64_t>(ncontrib_, 1) * sizeof(uint32_t)));
    ECK(cudaMalloc((void**)&eq_, std::max<int64_t>(nel * nedof, 1) * sizeof(int32_t)));
    ECK(cudaMemcpy(pos_, pos.data(), npos_ * sizeof(int64_t), cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(cptr_, cptr.data(), (npos_ + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(contrib_, contrib.data(), ncontrib_ * sizeof(uint32_t), cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(eq_, eq.data(), nel * nedof * sizeof(int32_t), cudaMemcpyHostToDevice));
    return 0;
}

// One thread per LNZ position that receives element contributions: the sum
// in element order with separately rounded products (no FMA), like the
// host's SM(K) = SM(K) + s*EM(I,J) from SM(K) = 0.
__global__ void k_elem_assemble(const int64_t* pos, const int64_t* cptr, const uint32_t* contrib, int64_t npos,
                                const double* em, const double* scale, int nedof, double* lnz) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= npos) return;
    const int64_t nn = (int64_t)nedof * nedof;
    double acc = 0.0;
    for (int64_t c = cptr[i]; c < cptr[i + 1]; ++c) {
        const uint32_t w = contrib[c];
        const int64_t e = w >> 10;
        const int idx = (int)(w & 1023u);
        const double v = scale ? __dmul_rn(scale[e], em[idx]) : em[e * nn + idx];
        acc = __dadd_rn(acc, v);
    }
    lnz[pos[i]] = acc;
}

// One warp per element: lane i < nedof forms (dK_e u_e)_i, multiplies by
// lam_e(i) and the warp sums; constrained DOFs contribute nothing.
__global__ void k_elem_grad(const int32_t* eq, int64_t nel, int nedof, const double* u, const double* lam,
                            int64_t ld, int nrhs, const double* em, const double* dscale, double* grad) {
    extern __shared__ double s_em[];
    const int nn = nedof * nedof;
    if (dscale)
        for (int k = threadIdx.x; k < nn; k += blockDim.x) s_em[k] = em[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    if (e >= nel) return;
    const double* K = dscale ? s_em : em + e * (int64_t)nn;
    const int32_t myeq = lane < nedof ? eq[e * nedof + lane] : -1;
    double total = 0.0;
    for (int q = 0; q < nrhs; ++q) {
        const double ui = myeq >= 0 ? u[myeq + q * ld] : 0.0;
        double t = 0.0;
        for (int j = 0; j < nedof; ++j) {
            const double uj = __shfl_sync(0xffffffffu, ui, j);
            if (lane < nedof) t += K[lane + j * nedof] * uj;
        }
        double v = myeq >= 0 ? lam[myeq + q * ld] * t : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        total += v;
    }
    if (lane == 0) grad[e] = -(dscale ? dscale[e] : 1.0) * total;
}

int Elements::assemble(double* d_sm, const double* d_em, const double* d_scale, cudaStream_t s) {
    ECK(cudaMemsetAsync(d_sm, 0, (neq_ + nzerol_) * sizeof(double), s));
    if (npos_ > 0)
        k_elem_assemble<<<(int)((npos_ + 255) / 256), 256, 0, s>>>(pos_, cptr_, contrib_, npos_, d_em, d_scale,
                                                                   (int)nedof_, d_sm + neq_);
    ECK(cudaGetLastError());
    return 0;
}

int Elements::grad(const double* d_u, const double* d_lam, int64_t ld, int64_t nrhs, const double* d_em,
                   const double* d_dscale, double* d_grad, cudaStream_t s) {
    if (ld < neq_ || nrhs < 1) return -2;
    if (nel_ > 0) {
        const size_t smem = d_dscale ? nedof_ * nedof_ * sizeof(double) : 0;
        k_elem_grad<<<(int)((nel_ * 32 + 255) / 256), 256, smem, s>>>(eq_, nel_, (int)nedof_, d_u, d_lam, ld,
                                                                      (int)nrhs, d_em, d_dscale, d_grad);
    }
    ECK(cudaGetLastError());
    return 0;
}

}  // namespace sprb
