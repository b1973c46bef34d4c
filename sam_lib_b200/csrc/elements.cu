// Element assembly (SPRADM/SPRAD2 as a gather), the hex8 element stiffness
// and the adjoint element gradient on the device.
#include "elements.h"

#include <algorithm>
#include <vector>

namespace sprb {

#define ECK(x)                                \
    do {                                      \
        if ((x) != cudaSuccess) return -4;    \
    } while (0)

void Elements::Gather::release() {
    cudaFree(pos);
    cudaFree(cptr);
    cudaFree(contrib);
    cudaFree(kind);
    cudaFree(jp);
    cudaFree(ip);
    *this = Gather();
}

Elements::~Elements() {
    sm_.release();
    sv_.release();
    cudaFree(eq_);
    cudaFree(enodes_);
}

// Groups the (target, record) pairs by target, keeping the visiting order
// inside each group, and uploads the plan.  The low 32 bits of a record are
// the contribution word, the high 32 bits its index into jp/ip/kind.
int Elements::upload(Gather& g, std::vector<std::pair<int64_t, uint64_t>>& pc, const std::vector<int32_t>& jp,
                     const std::vector<int32_t>& ip, const std::vector<uint8_t>& kind, bool weighted) {
    std::stable_sort(pc.begin(), pc.end(),
                     [](const std::pair<int64_t, uint64_t>& a, const std::pair<int64_t, uint64_t>& b) {
                         return a.first < b.first;
                     });
    std::vector<int64_t> pos, cptr;
    std::vector<uint32_t> contrib(pc.size());
    std::vector<uint8_t> k2(weighted ? pc.size() : 0);
    std::vector<int32_t> jp2(weighted ? pc.size() : 0), ip2(weighted ? pc.size() : 0);
    for (size_t i = 0; i < pc.size(); ++i) {
        if (i == 0 || pc[i].first != pc[i - 1].first) {
            pos.push_back(pc[i].first);
            cptr.push_back((int64_t)i);
        }
        contrib[i] = (uint32_t)pc[i].second;
        if (weighted) {
            const size_t a = (size_t)(pc[i].second >> 32);
            k2[i] = kind[a];
            jp2[i] = jp[a];
            ip2[i] = ip[a];
        }
    }
    cptr.push_back((int64_t)pc.size());
    g.npos = (int64_t)pos.size();
    g.ncontrib = (int64_t)pc.size();
    const size_t nc = std::max<size_t>(pc.size(), 1);
    ECK(cudaMalloc((void**)&g.pos, std::max<int64_t>(g.npos, 1) * sizeof(int64_t)));
    ECK(cudaMalloc((void**)&g.cptr, (g.npos + 1) * sizeof(int64_t)));
    ECK(cudaMalloc((void**)&g.contrib, nc * sizeof(uint32_t)));
    ECK(cudaMemcpy(g.pos, pos.data(), g.npos * sizeof(int64_t), cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(g.cptr, cptr.data(), (g.npos + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
    ECK(cudaMemcpy(g.contrib, contrib.data(), pc.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    if (weighted) {
        ECK(cudaMalloc((void**)&g.kind, nc));
        ECK(cudaMalloc((void**)&g.jp, nc * sizeof(int32_t)));
        ECK(cudaMalloc((void**)&g.ip, nc * sizeof(int32_t)));
        ECK(cudaMemcpy(g.kind, k2.data(), pc.size(), cudaMemcpyHostToDevice));
        ECK(cudaMemcpy(g.jp, jp2.data(), pc.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
        ECK(cudaMemcpy(g.ip, ip2.data(), pc.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    }
    return 0;
}

int Elements::open(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa, const int64_t* meqn,
                   const int64_t* madof, const int64_t* mpmnpc, const int64_t* mmnpc, int64_t nel,
                   int64_t nedof, const int64_t* mpmceq, const int64_t* mmceq, int64_t nceq) {
    if (nedof < 1 || nedof > 32 || nel < 0 || nel >= (int64_t(1) << 22) || nceq < 0) return -2;
    if (nceq > 0 && (!mpmceq || !mmceq || mpmceq[nceq] - 1 >= (int64_t(1) << 31))) return -2;
    neq_ = mspar[7];
    nzerol_ = mspar[15];
    nel_ = nel;
    nedof_ = nedof;
    const LnzIndex<int64_t> lx(mspar, mtrees, msifa);
    // equation map of every element (the adjoint gradient) and its nodes
    std::vector<int32_t> eq((size_t)nel * nedof);
    std::vector<int32_t> en((size_t)nel * 8);
    bool hex = nedof == 24;
    for (int64_t e = 0; e < nel; ++e) {
        int64_t nd = 0;
        if (mpmnpc[e + 1] - mpmnpc[e] != 8) hex = false;
        for (int64_t p = mpmnpc[e]; p < mpmnpc[e + 1]; ++p) {
            const int64_t node = mmnpc[p - 1];
            if (madof[node] - madof[node - 1] != 3) hex = false;
            if (hex) en[e * 8 + (p - mpmnpc[e])] = (int32_t)(node - 1);
            for (int64_t d = madof[node - 1]; d < madof[node]; ++d) {
                if (nd >= nedof) return -3;
                const int64_t q = meqn[d - 1];
                eq[e * nedof + nd++] = q >= 1 ? (int32_t)(q - 1) : -1;
            }
        }
        if (nd != nedof) return -3;
    }
    // the additions of SPRADM, in its order
    std::vector<std::pair<int64_t, uint64_t>> pcm, pcv;
    pcm.reserve((size_t)nel * nedof * (nedof + 1) / 2);
    std::vector<int32_t> jpv, ipv;
    std::vector<uint8_t> kv;
    const int rc = for_each_contribution(
        lx, meqn, madof, mpmnpc, mmnpc, mpmceq, mmceq, nceq, nel, nedof, true, nceq > 0,
        [&](bool to_sv, int64_t target, int64_t e, int64_t idx, int kind, int64_t jp, int64_t ip) {
            const uint64_t word = (uint64_t)((e << 10) | idx) | ((uint64_t)kv.size() << 32);
            if (nceq > 0) {
                kv.push_back((uint8_t)kind);
                jpv.push_back((int32_t)jp);
                ipv.push_back((int32_t)ip);
            }
            (to_sv ? pcv : pcm).emplace_back(target, word);
        });
    if (rc != 0) return rc;
    if (kv.size() >= (size_t(1) << 32)) return -2;
    int r = upload(sm_, pcm, jpv, ipv, kv, nceq > 0);
    if (r == 0 && nceq > 0) r = upload(sv_, pcv, jpv, ipv, kv, true);
    if (r != 0) return r;
    npos_ = sm_.npos;
    ncontrib_ = sm_.ncontrib;
    ECK(cudaMalloc((void**)&eq_, std::max<int64_t>(nel * nedof, 1) * sizeof(int32_t)));
    ECK(cudaMemcpy(eq_, eq.data(), nel * nedof * sizeof(int32_t), cudaMemcpyHostToDevice));
    if (hex && nel > 0) {
        ECK(cudaMalloc((void**)&enodes_, nel * 8 * sizeof(int32_t)));
        ECK(cudaMemcpy(enodes_, en.data(), nel * 8 * sizeof(int32_t), cudaMemcpyHostToDevice));
    }
    return 0;
}

// One thread per target (LNZ position or SV index) that receives element
// contributions: the sum in SPRADM's order with separately rounded
// products (no FMA), like the host's SM(K) = SM(K) + w*EM(I,J) from SM(K) =
// 0.  kind == null: every contribution is a plain EM(I,J).
__global__ void k_elem_assemble(const int64_t* pos, const int64_t* cptr, const uint32_t* contrib,
                                const uint8_t* kind, const int32_t* jp, const int32_t* ip, int64_t npos,
                                const double* em, const double* scale, int nedof, const double* ttcc,
                                double* out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= npos) return;
    const int64_t nn = (int64_t)nedof * nedof;
    double acc = 0.0;
    for (int64_t c = cptr[i]; c < cptr[i + 1]; ++c) {
        const uint32_t w = contrib[c];
        const int64_t e = w >> 10;
        const int idx = (int)(w & 1023u);
        double v = scale ? __dmul_rn(scale[e], em[idx]) : em[e * nn + idx];
        if (kind && !contrib_value(kind[c], v, ttcc, jp[c], ip[c], &v)) continue;
        acc = __dadd_rn(acc, v);
    }
    out[pos[i]] = acc;
}

// Hex8 stiffness, kHexEpb elements per CTA of 256 threads.  Stage 1: one
// thread per (element, Gauss point) forms J_ij = sum_a dN_a/dxi_i x_a,j,
// det J and dN/dx = J^-1 dN/dxi for the 8 nodes.  Stage 2: one thread per
// (element, node a, node b) sums over the Gauss points the 3x3 block
//   K_ab,ij = det J (lam g_a,i g_b,j + mu g_a,j g_b,i + mu [i=j] g_a.g_b),
// the closed form of B_a^T D B_b for isotropic D.  Stage 3: the CTA's
// matrices leave shared memory in coalesced rows.
constexpr int kHexEpb = 4;

__global__ void __launch_bounds__(256) k_hex8(const int32_t* enodes, int64_t nel, const double* xyz,
                                              const double* E, double nu, double* em) {
    __shared__ double s_x[kHexEpb][8][3];
    __shared__ double s_g[kHexEpb][8][8][3];
    __shared__ double s_w[kHexEpb][8];
    __shared__ double s_k[kHexEpb * 576];
    const int t = threadIdx.x;
    const int64_t e0 = (int64_t)blockIdx.x * kHexEpb;
    if (t < kHexEpb * 24) {
        const int le = t / 24, a = (t % 24) / 3, d = t % 3;
        const int64_t e = e0 + le;
        s_x[le][a][d] = e < nel ? xyz[(int64_t)enodes[e * 8 + a] * 3 + d] : (a == 0 ? 0.0 : 1.0);
    }
    __syncthreads();
    if (t < kHexEpb * 8) {
        const int le = t >> 3, gp = t & 7;
        // corners (0,0,0) (1,0,0) (1,1,0) (0,1,0) (0,0,1) (1,0,1) (1,1,1) (0,1,1) as signs
        const double cx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
        const double cy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
        const double cz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
        const double g = 1.0 / sqrt(3.0);
        const double xi = (gp & 1) ? g : -g, eta = (gp & 2) ? g : -g, zeta = (gp & 4) ? g : -g;
        double dn[8][3];
        double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int a = 0; a < 8; ++a) {
            dn[a][0] = cx[a] * (1 + eta * cy[a]) * (1 + zeta * cz[a]) / 8;
            dn[a][1] = cy[a] * (1 + xi * cx[a]) * (1 + zeta * cz[a]) / 8;
            dn[a][2] = cz[a] * (1 + xi * cx[a]) * (1 + eta * cy[a]) / 8;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) J[i][j] += dn[a][i] * s_x[le][a][j];
        }
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        const double r = 1.0 / det;
        // J^-1 = adj(J) / det, adj(J)_ij = cofactor_ji
        const double inv[3][3] = {
            {c00 * r, (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * r, (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * r},
            {c01 * r, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * r, (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * r},
            {c02 * r, (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * r, (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * r}};
#pragma unroll
        for (int a = 0; a < 8; ++a)
#pragma unroll
            for (int i = 0; i < 3; ++i)
                s_g[le][gp][a][i] = inv[i][0] * dn[a][0] + inv[i][1] * dn[a][1] + inv[i][2] * dn[a][2];
        s_w[le][gp] = det;
    }
    __syncthreads();
    {
        const int le = t >> 6, a = (t >> 3) & 7, b = t & 7;
        const int64_t e = e0 + le;
        const double Ee = e < nel ? E[e] : 0.0;
        const double lam = Ee * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
        const double mu = Ee / (2.0 * (1.0 + nu));
        double k[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
        for (int gp = 0; gp < 8; ++gp) {
            const double* ga = s_g[le][gp][a];
            const double* gb = s_g[le][gp][b];
            const double w = s_w[le][gp];
            const double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    k[i][j] += w * (lam * (ga[i] * gb[j]) + mu * (ga[j] * gb[i]) + (i == j ? mu * dot : 0.0));
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) s_k[le * 576 + (3 * a + i) + 24 * (3 * b + j)] = k[i][j];
    }
    __syncthreads();
    const int64_t lim = (nel - e0 < kHexEpb ? nel - e0 : kHexEpb) * 576;
    for (int64_t q = t; q < lim; q += 256) em[e0 * 576 + q] = s_k[q];
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

int Elements::assemble(double* d_sm, const double* d_em, const double* d_scale, cudaStream_t s, double* d_sv,
                       const double* d_ttcc) {
    if ((sm_.kind || sv_.kind) && !d_ttcc) return -2;
    if (d_sm) {
        ECK(cudaMemsetAsync(d_sm, 0, (neq_ + nzerol_) * sizeof(double), s));
        if (sm_.npos > 0)
            k_elem_assemble<<<(int)((sm_.npos + 255) / 256), 256, 0, s>>>(
                sm_.pos, sm_.cptr, sm_.contrib, sm_.kind, sm_.jp, sm_.ip, sm_.npos, d_em, d_scale, (int)nedof_,
                d_ttcc, d_sm + neq_);
    }
    if (d_sv) {
        ECK(cudaMemsetAsync(d_sv, 0, std::max<int64_t>(neq_, 1) * sizeof(double), s));
        if (sv_.npos > 0)
            k_elem_assemble<<<(int)((sv_.npos + 255) / 256), 256, 0, s>>>(
                sv_.pos, sv_.cptr, sv_.contrib, sv_.kind, sv_.jp, sv_.ip, sv_.npos, d_em, d_scale, (int)nedof_,
                d_ttcc, d_sv);
    }
    ECK(cudaGetLastError());
    return 0;
}

int Elements::hex8(const double* d_xyz, const double* d_E, double nu, double* d_em, cudaStream_t s) {
    if (!enodes_) return nel_ == 0 ? 0 : -2;
    const int64_t blocks = (nel_ + kHexEpb - 1) / kHexEpb;
    k_hex8<<<(unsigned)blocks, 256, 0, s>>>(enodes_, nel_, d_xyz, d_E, nu, d_em);
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
