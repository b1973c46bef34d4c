// Execution plan of the GPU numeric phase (see plan.h).
#include "plan.h"
#include "smhash.h"

#include <thread>

#include <algorithm>
#include <cmath>
#include <map>

namespace sprb {

namespace {

// First-fit allocator over a linear arena, in units of doubles.  Blocks are
// aligned to 32 doubles (256 bytes) so every front starts on a TMA/vector
// friendly boundary.
class Arena {
public:
    int64_t alloc(int64_t n) {
        n = (n + 31) / 32 * 32;
        if (n == 0) n = 32;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                int64_t off = it->first;
                int64_t rest = it->second - n;
                free_.erase(it);
                if (rest > 0) free_[off + n] = rest;
                return off;
            }
        }
        int64_t off = top_;
        top_ += n;
        peak_ = std::max(peak_, top_);
        return off;
    }
    void release(int64_t off, int64_t n) {
        n = (n + 31) / 32 * 32;
        if (n == 0) n = 32;
        auto it = free_.emplace(off, n).first;
        // coalesce with the next block
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        // coalesce with the previous block
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
                it = pv;
            }
        }
        // shrink the top
        if (it->first + it->second == top_) {
            top_ = it->first;
            free_.erase(it);
        }
    }
    int64_t peak() const { return peak_; }

private:
    std::map<int64_t, int64_t> free_;
    int64_t top_ = 0;
    int64_t peak_ = 0;
};

inline int32_t round_up4(int32_t x) { return (x + 3) / 4 * 4; }

}  // namespace

int build_plan(const int64_t* mspar, const int64_t* mtrees, const int64_t* msifa, Plan& P) {
    // Pointer conventions of SPRFC1 (src/SPR/sprfc1.f:165-196).
    P.neq = mspar[7];
    P.nsuper = mspar[10];
    P.maxsup = mspar[12];
    P.mfront = mspar[13];
    P.nofsub = mspar[14];
    P.nzerol = mspar[15];
    const int64_t ns = P.nsuper;
    if (ns <= 0 || P.neq <= 0 || mspar[44] < 1 || mspar[45] < 1 || mspar[46] < 1 || mspar[47] < 1)
        return -2;
    const int64_t* xsuper = mtrees + (mspar[44] - 1);
    const int64_t* xsibl = xsuper + (ns + 1);
    const int64_t* sibl = xsuper + 2 * (ns + 1);
    const int64_t* xlindx = mtrees + (mspar[45] - 1);
    const int64_t* lindx = msifa + (mspar[46] - 1);
    const int64_t* xlnz = msifa + (mspar[47] - 1);
    const int64_t* supsup = xlindx + (ns + 1);          // sprfc1.f:183
    const bool lpar57 = mspar[56] > 0;

    P.retained.assign(ns, 0);
    P.any_retained = false;
    if (lpar57)
        for (int64_t js = 0; js < ns; ++js)
            if (supsup[js] > 0) {
                P.retained[js] = 1;
                P.any_retained = true;
            }
    P.fst.resize(ns);
    P.S.resize(ns);
    P.F.resize(ns);
    P.parent.assign(ns, -1);
    P.level.assign(ns, 0);
    P.lnz_off.resize(ns);
    P.lindx_off.resize(ns);
    P.child_ptr.assign(ns + 1, 0);
    P.factor_flops = 0.0;
    P.solve_flops = 0.0;
    for (int64_t js = 0; js < ns; ++js) {
        P.fst[js] = (int32_t)(xsuper[js] - 1);
        P.S[js] = (int32_t)(xsuper[js + 1] - xsuper[js]);
        P.F[js] = (int32_t)(xlindx[js + 1] - xlindx[js]);
        P.lnz_off[js] = xlnz[js] - 1;
        P.lindx_off[js] = xlindx[js] - 1;
        if (P.S[js] <= 0 || P.F[js] < P.S[js]) return -2;
        if (P.retained[js]) continue;                  // sprtrs.f:1956
        const double s = P.S[js], f = P.F[js];
        // RINFO(3) and RINFO(4) per supernode, src/SPR/sprtrs.f:1961-1980
        P.factor_flops += ((f * f) + 2.0 * f) * s - 2.0 * (1.0 + f) * (s * (s + 1.0) / 2.0) +
                          s * (s + 1.0) * (2.0 * s + 1.0) / 6.0;
        P.solve_flops += f * s - s * (s - 1.0) / 2.0 - s;
    }
    P.solve_flops = 2.0 * P.solve_flops + (double)P.neq;
    // children (SIBL order) and parents
    P.child.clear();
    for (int64_t js = 0; js < ns; ++js) {
        P.child_ptr[js] = (int32_t)P.child.size();
        for (int64_t k = xsibl[js]; k < xsibl[js + 1]; ++k) {
            int64_t c = sibl[k - 1] - 1;
            if (c < 0 || c >= js) return -2;   // postorder: children precede parents
            P.child.push_back((int32_t)c);
            P.parent[c] = (int32_t)js;
        }
    }
    P.child_ptr[ns] = (int32_t)P.child.size();
    // rows (0-based)
    P.rows.resize(xlindx[ns] - 1);
    for (size_t i = 0; i < P.rows.size(); ++i) P.rows[i] = (int32_t)(lindx[i] - 1);
    // levels: leaves 0, parent = 1 + max(children)
    int32_t nlev = 0;
    for (int64_t js = 0; js < ns; ++js) {
        int32_t lv = 0;
        for (int32_t k = P.child_ptr[js]; k < P.child_ptr[js + 1]; ++k)
            lv = std::max(lv, P.level[P.child[k]] + 1);
        P.level[js] = lv;
        nlev = std::max(nlev, lv + 1);
    }
    // relative maps (SPRF12 merge) and the contribution lists
    P.rel_off.assign(ns, -1);
    P.rel.clear();
    P.rbase.assign(ns + 1, 0);
    for (int64_t js = 0; js < ns; ++js) P.rbase[js + 1] = P.rbase[js] + P.F[js];
    std::vector<int64_t> ccount(P.rbase[ns] + 1, 0);
    for (int64_t c = 0; c < ns; ++c) {
        const int32_t q = P.F[c] - P.S[c];
        const int32_t p = P.parent[c];
        if (q <= 0) continue;
        if (p < 0) return -2;                  // update rows without a parent
        P.rel_off[c] = (int64_t)P.rel.size();
        const int32_t* prow = &P.rows[P.lindx_off[p]];
        const int32_t* crow = &P.rows[P.lindx_off[c] + P.S[c]];
        int32_t sup = 0;
        for (int32_t t = 0; t < q; ++t) {
            while (sup < P.F[p] && prow[sup] < crow[t]) ++sup;
            if (sup >= P.F[p] || prow[sup] != crow[t]) return -4;   // not a subset
            P.rel.push_back(sup);
            ccount[P.rbase[p] + sup + 1]++;
            ++sup;
        }
    }
    P.cptr.assign(P.rbase[ns] + 1, 0);
    for (int64_t i = 0; i < P.rbase[ns]; ++i) P.cptr[i + 1] = P.cptr[i] + ccount[i + 1];
    P.cchild.assign(P.cptr[P.rbase[ns]], 0);
    P.ct.assign(P.cptr[P.rbase[ns]], 0);
    {
        std::vector<int64_t> fill(P.cptr.begin(), P.cptr.end() - 1);
        // children in the reference's assembly order: last sibling first (sprfc1.f:534)
        for (int64_t p = 0; p < ns; ++p) {
            for (int32_t k = P.child_ptr[p + 1] - 1; k >= P.child_ptr[p]; --k) {
                const int32_t c = P.child[k];
                const int32_t q = P.F[c] - P.S[c];
                for (int32_t t = 0; t < q; ++t) {
                    const int32_t j = P.rel[P.rel_off[c] + t];
                    const int64_t pos = fill[P.rbase[p] + j]++;
                    P.cchild[pos] = c;
                    P.ct[pos] = t;
                }
            }
        }
    }
    // arena layout, level by level
    P.buf_off.assign(ns, 0);
    P.buf_ld.assign(ns, 0);
    P.upd_off.assign(ns, 0);
    P.levels.assign(nlev, LevelPlan());
    std::vector<std::vector<int32_t>> bylev(nlev);
    for (int64_t js = 0; js < ns; ++js) bylev[P.level[js]].push_back((int32_t)js);
    std::vector<int64_t> buf_size(ns, 0);
    Arena arena;
    P.any_large = false;
    for (int32_t L = 0; L < nlev; ++L) {
        LevelPlan& lp = P.levels[L];
        std::vector<int32_t> nodes = bylev[L];
        // big buffers first: less fragmentation
        std::stable_sort(nodes.begin(), nodes.end(),
                         [&](int32_t a, int32_t b) { return P.F[a] > P.F[b]; });
        for (int32_t js : nodes) {
            const int32_t f = P.F[js], s = P.S[js], q = f - s;
            if (f <= kSmallMaxF) {
                lp.small_nodes.push_back(js);
                lp.small_maxF = std::max(lp.small_maxF, f);
                P.buf_ld[js] = std::max(q, 1);
                buf_size[js] = (int64_t)q * q;
                P.buf_off[js] = arena.alloc(buf_size[js]);
                P.upd_off[js] = P.buf_off[js];
            } else {
                lp.large_nodes.push_back(js);
                P.any_large = true;
                const int32_t ld = round_up4(f);
                P.buf_ld[js] = ld;
                buf_size[js] = (int64_t)ld * f;
                P.buf_off[js] = arena.alloc(buf_size[js]);
                P.upd_off[js] = P.buf_off[js] + (int64_t)s * ld + s;
            }
        }
        // small_nodes are in decreasing F: cut them into size classes
        {
            auto cls = [](int32_t f) { return f <= 64 ? 0 : f <= 96 ? 1 : f <= 128 ? 2 : 3; };
            for (int32_t k = 0; k < (int32_t)lp.small_nodes.size();) {
                const int32_t c = cls(P.F[lp.small_nodes[k]]);
                int32_t e = k;
                while (e < (int32_t)lp.small_nodes.size() && cls(P.F[lp.small_nodes[e]]) == c) ++e;
                lp.small_classes.push_back(LevelPlan::SmallClass{k, e - k, P.F[lp.small_nodes[k]]});
                k = e;
            }
        }
        // after this level is assembled, its children are no longer needed
        for (int32_t js : nodes)
            for (int32_t k = P.child_ptr[js]; k < P.child_ptr[js + 1]; ++k) {
                const int32_t c = P.child[k];
                arena.release(P.buf_off[c], buf_size[c]);
            }
    }
    P.arena_doubles = arena.peak();
    P.xinv_off.assign(ns, -1);
    P.xinv_doubles = 0;
    for (int64_t js = 0; js < ns; ++js)
        if (P.F[js] > kSmallMaxF) {
            const int64_t nsb = (P.S[js] + kSolveBlock - 1) / kSolveBlock;
            const int64_t last = P.S[js] - (nsb - 1) * kSolveBlock;
            P.xinv_off[js] = P.xinv_doubles;
            P.xinv_doubles += ((nsb - 1) * kSolveBlock * kSolveBlock + last * last + 31) / 32 * 32;
        }
    P.linv_off.assign(ns, -1);
    P.linv_doubles = 0;
    for (int64_t js = 0; js < ns; ++js)
        if (P.F[js] > kSmallMaxF) {
            P.linv_off[js] = P.linv_doubles;
            P.linv_doubles += (int64_t)((P.S[js] + kNB - 1) / kNB) * kNB * kNB;
        }
    // ---- batched launches of the large path
    P.jobs.clear();
    P.alt.clear();
    P.rect_off.assign(ns, 0);
    P.rect_entries = 0;
    P.fwd_off.assign(ns, 0);
    P.fwd_entries = 0;
    auto open_launch = [&](Launch& l) { l.job_begin = (int64_t)P.jobs.size(); l.ntasks = 0; };
    auto add_job = [&](Launch& l, Job j, int64_t ntask, bool keep_empty = false) {
        if (ntask <= 0 && !keep_empty) return;
        j.task0 = l.ntasks;
        P.jobs.push_back(j);
        l.ntasks += std::max<int64_t>(ntask, 0);
    };
    auto close_launch = [&](Launch& l) { l.job_count = (int64_t)P.jobs.size() - l.job_begin; };
    P.gemm_flops = 0.0;
    P.tc_flops = 0.0;
    P.slab_rows = 0;
    P.slab_rows_far = 0;
    P.small_flops = 0.0;
    for (int64_t js = 0; js < ns; ++js)
        if (P.F[js] <= kSmallMaxF) {
            const double s = P.S[js], f = P.F[js];
            P.small_flops += ((f * f) + 2.0 * f) * s - 2.0 * (1.0 + f) * (s * (s + 1.0) / 2.0) +
                             s * (s + 1.0) * (2.0 * s + 1.0) / 6.0;
        }
    // lower-triangle entries of rows [c0, r_end) x columns [c0, c_end), times 2K
    auto update_flops = [](int32_t c0, int32_t c_end, int32_t r_end, int32_t k) -> double {
        double e = 0.0;
        const double n = c_end - c0, r = r_end - c0;
        e = n * r - n * (n - 1.0) / 2.0;
        return 2.0 * e * k;
    };
    auto tiles_t = [](int32_t c0, int32_t c_end, int32_t r_end, int32_t t) -> int64_t {
        const int64_t nct = (c_end - c0 + t - 1) / t;
        const int64_t nr = (r_end - c0 + t - 1) / t;
        return nct * nr - nct * (nct - 1) / 2;
    };
    for (int32_t L = 0; L < nlev; ++L) {
        LevelPlan& lp = P.levels[L];
        if (lp.large_nodes.empty()) continue;
        open_launch(lp.assemble);
        for (int32_t js : lp.large_nodes)
            add_job(lp.assemble, Job{js, 0, P.F[js], P.F[js], 0, 0, 0}, P.F[js]);
        close_launch(lp.assemble);
        // elimination, Schur updates and the solve steps: retained fronts excluded
        lp.elim_nodes.clear();
        for (int32_t js : lp.large_nodes)
            if (!P.retained[js]) lp.elim_nodes.push_back(js);
        const std::vector<int32_t>& elim = lp.elim_nodes;
        int32_t smax = 0;
        for (int32_t js : elim) smax = std::max(smax, P.S[js]);
        const int32_t nsteps = (smax + kNB - 1) / kNB;
        lp.panel.assign(nsteps, Launch());
        lp.update.assign(nsteps, std::vector<Launch>());
        lp.fsolve.assign(nsteps, Launch());
        lp.bsolve.assign(nsteps, Launch());
        // Schur-update jobs of one step, split into a big-tile and a small-tile launch
        auto emit_updates = [&](std::vector<Job>& jl, std::vector<Launch>& out) {
            for (int pass = 0; pass < 2; ++pass) {
                const int32_t tile = pass == 0 ? kTileBig : kTile;
                Launch l;
                l.tile = tile;
                open_launch(l);
                for (const Job& j : jl) {
                    const bool big = (j.r_end - j.c0) >= 4 * kTileBig;
                    if (big != (pass == 0)) continue;
                    add_job(l, j, tiles_t(j.c0, j.c_end, j.r_end, tile));
                }
                close_launch(l);
                l.tile = tile;
                if (l.ntasks <= 0) continue;
                if (pass == 1) {
                    // the same jobs in kTileTiny tiles, for the tile autotuner
                    Launch a;
                    open_launch(a);
                    for (const Job& j : jl)
                        if ((j.r_end - j.c0) < 4 * kTileBig) add_job(a, j, tiles_t(j.c0, j.c_end, j.r_end, kTileTiny));
                    close_launch(a);
                    a.tile = kTileTiny;
                    l.alt = (int32_t)P.alt.size();
                    P.alt.push_back(a);
                }
                out.push_back(l);
            }
        };
        // the far and K = S updates for the tensor-core path: slabs of W = L D
        // and L as FP32 hi/lo pairs (4 arrays of K blocks of [rows][32])
        auto emit_tc = [&](std::vector<Job> jl, std::vector<TcLaunch>& out, int64_t& slab_max) {
            if (jl.empty()) return;
            int64_t rows = 0;
            for (Job& j : jl) {
                const int64_t np = (int64_t)(j.r_end - j.c0 + kTcTile - 1) / kTcTile * kTcTile;
                const int64_t nkb = (j.k_hi - j.k_lo + kTcBK - 1) / kTcBK;
                j.slab = rows;
                rows += 4 * nkb * np;
            }
            TcLaunch t;
            open_launch(t.split);
            for (const Job& j : jl) {
                const int64_t np = (int64_t)(j.r_end - j.c0 + kTcTile - 1) / kTcTile * kTcTile;
                const int64_t nkb = (j.k_hi - j.k_lo + kTcBK - 1) / kTcBK;
                add_job(t.split, j, (np / 32) * nkb);
            }
            close_launch(t.split);
            open_launch(t.gemm);
            for (const Job& j : jl) add_job(t.gemm, j, tiles_t(j.c0, j.c_end, j.r_end, kTcTile));
            close_launch(t.gemm);
            t.gemm.tile = kTcTile;
            slab_max = std::max(slab_max, rows);
            out.push_back(t);
        };
        lp.far.assign(nsteps, std::vector<Launch>());
        lp.ahead.assign(nsteps, std::vector<Launch>());
        lp.next_tc.assign(nsteps, std::vector<TcLaunch>());
        lp.next_flops.assign(nsteps, 0.0);
        lp.far_tc.assign(nsteps, std::vector<TcLaunch>());
        lp.far_flops.assign(nsteps, 0.0);
        for (int32_t st = 0; st < nsteps; ++st) {
            const int32_t k0 = st * kNB;
            open_launch(lp.panel[st]);
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (k0 >= s) continue;
                const int32_t nb = std::min(kNB, s - k0);
                const int64_t nrb = (f - (k0 + nb) + kTRSMRows - 1) / kTRSMRows;
                add_job(lp.panel[st], Job{js, k0 + nb, k0 + nb, f, k0, k0 + nb, 0}, nrb, true);
            }
            close_launch(lp.panel[st]);
            std::vector<Job> jl, jahead, jfar;
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (k0 >= s) continue;
                const int32_t nb = std::min(kNB, s - k0);
                const int32_t c0 = k0 + nb;
                const int32_t sp0 = (k0 / kSuperPanel) * kSuperPanel;
                const int32_t sp1 = std::min(sp0 + kSuperPanel, s);
                if (c0 < sp1) {                                     // inside the super-panel
                    // the next panel's columns on the panel chain; the ones
                    // after it beside the next diagonal block and TRSM
                    const int32_t c1 = std::min(c0 + kNB, sp1);
                    jl.push_back(Job{js, c0, c1, f, k0, c0, 0});
                    if (c1 < sp1) jahead.push_back(Job{js, c1, sp1, f, k0, c0, 0});
                    P.gemm_flops += update_flops(c0, sp1, f, nb);
                }
                if (c0 == sp1 && sp1 < s) {                          // trailing, K = kSuperPanel
                    // the next super-panel's columns now; the columns beyond
                    // it on the side stream, overlapping that super-panel
                    const int32_t sp2 = std::min(sp1 + kSuperPanel, s);
                    jl.push_back(Job{js, sp1, sp2, f, sp0, sp1, 0});
                    P.gemm_flops += update_flops(sp1, sp2, f, sp1 - sp0);
                    lp.next_flops[st] += update_flops(sp1, sp2, f, sp1 - sp0);
                    if (sp2 < s) {
                        jfar.push_back(Job{js, sp2, s, f, sp0, sp1, 0});
                        P.gemm_flops += update_flops(sp2, s, f, sp1 - sp0);
                        P.tc_flops += update_flops(sp2, s, f, sp1 - sp0);
                        lp.far_flops[st] += update_flops(sp2, s, f, sp1 - sp0);
                    }
                }
            }
            emit_updates(jl, lp.update[st]);
            if (lp.next_flops[st] > 0.0) emit_tc(jl, lp.next_tc[st], P.slab_rows);
            emit_updates(jahead, lp.ahead[st]);
            emit_updates(jfar, lp.far[st]);
            emit_tc(jfar, lp.far_tc[st], P.slab_rows_far);
            open_launch(lp.fsolve[st]);
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (k0 >= s) continue;
                const int32_t nb = std::min(kNB, s - k0);
                const int64_t nrb = (f - (k0 + nb) + kTRSMRows - 1) / kTRSMRows;
                add_job(lp.fsolve[st], Job{js, k0 + nb, k0 + nb, f, k0, k0 + nb, 0}, 1 + nrb);
            }
            close_launch(lp.fsolve[st]);
            open_launch(lp.bsolve[st]);
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (k0 >= s) continue;
                const int32_t nb = std::min(kNB, s - k0);
                add_job(lp.bsolve[st], Job{js, 0, k0, f, k0, k0 + nb, 0}, 1 + (k0 + kBwdCols - 1) / kBwdCols);
            }
            close_launch(lp.bsolve[st]);
        }
        const int32_t nsb = (smax + kSolveBlock - 1) / kSolveBlock;
        lp.fs_upd.assign(nsb, Launch());
        lp.bs_upd.assign(nsb, Launch());
        lp.blk_mv.assign(nsb, Launch());
        for (int32_t sb = 0; sb < nsb; ++sb) {
            const int32_t k0 = sb * kSolveBlock;
            open_launch(lp.blk_mv[sb]);
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (k0 >= s) continue;
                const int32_t k1 = std::min(k0 + kSolveBlock, s);
                add_job(lp.blk_mv[sb], Job{js, k0, k1, f, k0, k1, 0}, (k1 - k0 + 31) / 32);
            }
            close_launch(lp.blk_mv[sb]);
            open_launch(lp.fs_upd[sb]);
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (k0 >= s) continue;
                const int32_t k1 = std::min(k0 + kSolveBlock, s);
                // rows [k1, S) of the diagonal part; rows [S, F) go to the rectangle launch
                add_job(lp.fs_upd[sb], Job{js, k1, k1, s, k0, k1, 0}, (s - k1 + kSolveRows - 1) / kSolveRows, true);
            }
            close_launch(lp.fs_upd[sb]);
            open_launch(lp.bs_upd[sb]);
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (k0 >= s) continue;
                const int32_t k1 = std::min(k0 + kSolveBlock, s);
                add_job(lp.bs_upd[sb], Job{js, 0, k0, f, k0, k1, 0}, (k0 + kBwdCols - 1) / kBwdCols, true);
            }
            close_launch(lp.bs_upd[sb]);
        }
        open_launch(lp.rect);
        int64_t roff = 0, foff = 0;
        for (int32_t js : elim) {
            const int32_t s = P.S[js], f = P.F[js];
            if (f <= s) continue;
            const int64_t nrc = (f - s + kRectRows - 1) / kRectRows;
            const int64_t ncc = (s + kRectCols - 1) / kRectCols;
            P.rect_off[js] = roff;
            roff += nrc * s;
            P.fwd_off[js] = foff;
            foff += ncc * (f - s);
            add_job(lp.rect, Job{js, 0, s, f, (int32_t)nrc, (int32_t)ncc, 0}, nrc * ncc);
        }
        P.rect_entries = std::max(P.rect_entries, roff);
        P.fwd_entries = std::max(P.fwd_entries, foff);
        close_launch(lp.rect);
        open_launch(lp.rect_rows);
        for (int32_t js : elim) {
            const int32_t s = P.S[js], f = P.F[js];
            if (f > s) add_job(lp.rect_rows, Job{js, s, f, f, 0, 0, 0}, f - s);
        }
        close_launch(lp.rect_rows);
        {
            std::vector<Job> jl;
            for (int32_t js : elim) {
                const int32_t s = P.S[js], f = P.F[js];
                if (f > s) {
                    jl.push_back(Job{js, s, f, f, 0, s, 0});
                    P.gemm_flops += update_flops(s, f, f, s);
                    P.tc_flops += update_flops(s, f, f, s);
                    lp.outer_flops += update_flops(s, f, f, s);
                }
            }
            lp.outer.clear();
            emit_updates(jl, lp.outer);
            lp.outer_tc.clear();
            emit_tc(jl, lp.outer_tc, P.slab_rows);
        }
        open_launch(lp.writeback);
        for (int32_t js : lp.large_nodes)
            add_job(lp.writeback, Job{js, 0, P.S[js], P.F[js], 0, 0, 0}, P.S[js]);
        close_launch(lp.writeback);
        const int32_t nst = (int32_t)lp.panel.size();
        lp.wb_sp.assign(nst, Launch());
        for (int32_t st = 0; st < nst; ++st) {
            open_launch(lp.wb_sp[st]);
            for (int32_t js : lp.elim_nodes) {
                const int32_t s = P.S[js], k0 = st * kNB;
                if (k0 >= s) continue;
                const int32_t k1 = std::min(k0 + kNB, s);
                if (k1 % kSuperPanel != 0 && k1 != s) continue;     // the step does not end a super-panel
                const int32_t sp0 = (k0 / kSuperPanel) * kSuperPanel;
                add_job(lp.wb_sp[st], Job{js, sp0, k1, P.F[js], 0, 0, 0}, k1 - sp0);
            }
            close_launch(lp.wb_sp[st]);
        }
    }
    // task -> job maps of every launch
    P.task_map.clear();
    auto build_map = [&](Launch& l) {
        l.map_begin = (int64_t)P.task_map.size();
        for (int64_t j = 0; j < l.job_count; ++j) {
            const int64_t t0 = P.jobs[l.job_begin + j].task0;
            const int64_t t1 = (j + 1 < l.job_count) ? P.jobs[l.job_begin + j + 1].task0 : l.ntasks;
            for (int64_t t = t0; t < t1; ++t) P.task_map.push_back((int32_t)j);
        }
    };
    for (Launch& l : P.alt) build_map(l);
    for (LevelPlan& lp : P.levels) {
        build_map(lp.assemble);
        build_map(lp.writeback);
        for (Launch& l : lp.wb_sp) build_map(l);
        build_map(lp.rect);
        build_map(lp.rect_rows);
        for (Launch& l : lp.panel) build_map(l);
        for (auto& v : lp.update)
            for (Launch& l : v) build_map(l);
        for (auto& v : lp.ahead)
            for (Launch& l : v) build_map(l);
        for (Launch& l : lp.outer) build_map(l);
        for (auto& v : lp.far)
            for (Launch& l : v) build_map(l);
        for (auto& v : lp.far_tc)
            for (TcLaunch& t : v) {
                build_map(t.split);
                build_map(t.gemm);
            }
        for (auto& v : lp.next_tc)
            for (TcLaunch& t : v) {
                build_map(t.split);
                build_map(t.gemm);
            }
        for (TcLaunch& t : lp.outer_tc) {
            build_map(t.split);
            build_map(t.gemm);
        }
        for (Launch& l : lp.fs_upd) build_map(l);
        for (Launch& l : lp.bs_upd) build_map(l);
        for (Launch& l : lp.blk_mv) build_map(l);
    }
    // triangle tasks of the solves: per level, block-major (every task's
    // dependencies, the lower blocks of its own front, come earlier)
    P.tri_off.assign(ns, -1);
    P.tri_flags = 0;
    P.tri_tasks.clear();
    for (LevelPlan& lp : P.levels) {
        std::vector<int32_t> fr;
        int32_t nbmax = 0;
        for (int32_t js : lp.elim_nodes) {
            if (P.F[js] <= kSmallMaxF) continue;
            fr.push_back(js);
            P.tri_off[js] = P.tri_flags;
            const int32_t nb = (P.S[js] + kNB - 1) / kNB;
            P.tri_flags += nb;
            nbmax = std::max(nbmax, nb);
        }
        lp.tri_begin = (int64_t)P.tri_tasks.size() / 2;
        for (int32_t b = 0; b < nbmax; ++b)
            for (int32_t js : fr)
                if (b * kNB < P.S[js]) {
                    P.tri_tasks.push_back(js);
                    P.tri_tasks.push_back(b);
                }
        lp.tri_count = (int64_t)P.tri_tasks.size() / 2 - lp.tri_begin;
    }
    open_launch(P.inv_blocks);
    for (int64_t js = 0; js < ns; ++js) {
        if (P.F[js] <= kSmallMaxF || P.retained[js]) continue;
        for (int32_t k0 = 0; k0 < P.S[js]; k0 += kSolveBlock)
            add_job(P.inv_blocks, Job{(int32_t)js, k0, std::min(k0 + kSolveBlock, P.S[js]), P.F[js], k0,
                                      std::min(k0 + kSolveBlock, P.S[js]), 0}, 1);
    }
    close_launch(P.inv_blocks);
    return 0;
}

int64_t buffer_doubles(const Plan& P, int64_t js) {
    const int64_t f = P.F[js], s = P.S[js];
    return (f <= kSmallMaxF) ? (f - s) * (f - s) : (int64_t)P.buf_ld[js] * f;
}

// Every buffer inside the arena, and no two buffers that are live at the same
// level (from the node's own level to its parent's) overlap.
void check_plan(const Plan& P, int64_t& oob, int64_t& overlaps) {
    oob = 0;
    overlaps = 0;
    const int64_t ns = P.nsuper;
    for (int64_t js = 0; js < ns; ++js)
        if (P.buf_off[js] < 0 || P.buf_off[js] + buffer_doubles(P, js) > P.arena_doubles) ++oob;
    // index maps: a child's relative rows (SPRF12's LINDEX) lie in [0, F_p)
    // of its parent's rows, strictly increasing, and its column t lands in
    // parent column rel[t] exactly once in the contribution lists
    std::vector<int64_t> seen(P.rel.size(), 0);
    for (int64_t c = 0; c < ns; ++c) {
        const int32_t q = P.F[c] - P.S[c];
        if (q <= 0) continue;
        const int32_t p = P.parent[c];
        if (p < 0 || P.rel_off[c] < 0 || P.rel_off[c] + q > (int64_t)P.rel.size()) {
            ++oob;
            continue;
        }
        for (int32_t t = 0; t < q; ++t) {
            const int32_t r = P.rel[P.rel_off[c] + t];
            if (r < 0 || r >= P.F[p] || (t > 0 && r <= P.rel[P.rel_off[c] + t - 1])) ++oob;
        }
    }
    for (int64_t p = 0; p < ns; ++p)
        for (int32_t j = 0; j < P.F[p]; ++j)
            for (int64_t e = P.cptr[P.rbase[p] + j]; e < P.cptr[P.rbase[p] + j + 1]; ++e) {
                const int32_t c = P.cchild[e], t = P.ct[e];
                if (c < 0 || c >= ns || P.parent[c] != p || t < 0 || t >= P.F[c] - P.S[c] ||
                    P.rel[P.rel_off[c] + t] != j) {
                    ++oob;
                    continue;
                }
                ++seen[P.rel_off[c] + t];
            }
    for (int64_t k = 0; k < (int64_t)seen.size(); ++k)
        if (seen[k] != 1) ++oob;
    const int32_t nlev = (int32_t)P.levels.size();
    std::vector<std::vector<int32_t>> live(nlev);
    for (int64_t js = 0; js < ns; ++js) {
        const int32_t l0 = P.level[js];
        const int32_t l1 = P.parent[js] >= 0 ? P.level[P.parent[js]] : l0;
        for (int32_t L = l0; L <= l1; ++L) live[L].push_back((int32_t)js);
    }
    for (int32_t L = 0; L < nlev; ++L) {
        std::vector<std::pair<int64_t, int64_t>> iv;
        for (int32_t js : live[L]) {
            const int64_t n = buffer_doubles(P, js);
            if (n > 0) iv.emplace_back(P.buf_off[js], P.buf_off[js] + n);
        }
        std::sort(iv.begin(), iv.end());
        for (size_t k = 1; k < iv.size(); ++k)
            if (iv[k].first < iv[k - 1].second) ++overlaps;
    }
}

void check_coverage(const Plan& P, int64_t& fp64, int64_t& tc) {
    fp64 = tc = 0;
    const int64_t ns = P.nsuper;
    for (int which = 0; which < 2; ++which) {
        // per front: per column, the K intervals it receives
        std::vector<std::vector<std::vector<std::pair<int32_t, int32_t>>>> cov(ns);
        auto add = [&](const Launch& l) {
            for (int64_t j = 0; j < l.job_count; ++j) {
                const Job& jb = P.jobs[l.job_begin + j];
                auto& c = cov[jb.node];
                if (c.empty()) c.resize(P.F[jb.node]);
                for (int32_t col = jb.c0; col < jb.c_end; ++col) c[col].emplace_back(jb.k_lo, jb.k_hi);
            }
        };
        for (const LevelPlan& lp : P.levels) {
            for (const auto& v : lp.update)
                for (const Launch& l : v) add(l);
            for (const auto& v : lp.ahead)
                for (const Launch& l : v) add(l);
            if (which == 0) {
                for (const auto& v : lp.far)
                    for (const Launch& l : v) add(l);
                for (const Launch& l : lp.outer) add(l);
            } else {
                for (const auto& v : lp.far_tc)
                    for (const TcLaunch& t : v) add(t.gemm);
                for (const TcLaunch& t : lp.outer_tc) add(t.gemm);
            }
        }
        int64_t bad = 0;
        for (int64_t js = 0; js < ns; ++js) {
            if (P.F[js] <= kSmallMaxF) continue;
            const int32_t F = P.F[js], S = P.S[js];
            auto& c = cov[js];
            if (c.empty()) c.resize(F);
            for (int32_t col = 0; col < F; ++col) {
                // a retained front receives no update at all
                const int32_t want = P.retained[js] ? 0 : col < S ? (col / kNB) * kNB : S;
                auto& v = c[col];
                std::sort(v.begin(), v.end());
                int32_t at = 0;
                bool ok = true;
                for (const auto& iv : v) {
                    if (iv.first != at || iv.second <= iv.first) {
                        ok = false;
                        break;
                    }
                    at = iv.second;
                }
                if (!ok || at != want) ++bad;
            }
        }
        (which == 0 ? fp64 : tc) = bad;
    }
}


// ---------------------------------------------------------------------------
// Stream-schedule check of the factorisation (a race detector on the host).
//
// Replays the launch order of the factorisation of every level: per panel
// step the diagonal block + TRSM and the panel-chain updates on the main
// stream; inside a super-panel the update of the columns after the next
// panel on the look-ahead stream, forked by an event after the step's TRSM
// and joined before the next step's chain update; at the end of a
// super-panel the far columns' update on the side stream, forked by an event
// after the step's TRSM and joined before the next trailing update (every
// kSuperPanel / kNB steps) and before the K = S update.  Vector clocks give
// the happens-before order of the three streams.  Per large front it counts
//   * a panel whose columns have not received exactly the K ranges [0, k0)
//     from updates ordered before it, or that an unordered update writes;
//   * an update whose K panel columns are not final (diagonal block + TRSM
//     ordered before it);
//   * two updates on different streams that write a common element unordered;
//   * an update of the S columns not ordered before the write-back.
// tc: the far and K = S updates take the tensor-core path (split + product on
// the same stream as the FP64 launch they replace).  skip_join drops joins
// (bit 0: the far updates', bit 1: the look-ahead updates'), which must make
// the check fail wherever such launches exist.
// ---------------------------------------------------------------------------
namespace {
constexpr int kStreams = 3;          // 0 main, 1 side (far columns), 2 look-ahead
struct SchedOp {
    int stream;
    int64_t vc[kStreams];            // vector clock after the op
    int32_t c0, c_end, r0, r_end;    // written block (columns, rows)
    int32_t k_lo, k_hi;              // K range applied (updates)
    int kind;                        // 0 panel, 1 update, 2 write-back
};
bool hb(const SchedOp& a, const SchedOp& b) { return a.vc[a.stream] <= b.vc[a.stream]; }
}  // namespace

// number of tasks of job j of launch l
static int64_t job_tasks(const Plan& P, const Launch& l, int64_t j) {
    const int64_t t0 = P.jobs[l.job_begin + j].task0;
    const int64_t t1 = (j + 1 < l.job_count) ? P.jobs[l.job_begin + j + 1].task0 : l.ntasks;
    return t1 - t0;
}

// disjoint half-open ranges inside [0, cap): the number of ranges that are not
static int64_t range_faults(std::vector<std::pair<int64_t, int64_t>> iv, int64_t cap) {
    int64_t bad = 0;
    for (const auto& r : iv)
        if (r.first < 0 || r.second > cap) ++bad;
    std::sort(iv.begin(), iv.end());
    for (size_t k = 1; k < iv.size(); ++k)
        if (iv[k].first < iv[k - 1].second) ++bad;
    return bad;
}

int64_t check_solve_plan(const Plan& P, int plant, int64_t* tasks) {
    const int64_t ns = P.nsuper;
    // the two arrays a planted mistake changes, as copies
    std::vector<int32_t> tt = P.tri_tasks;
    std::vector<int64_t> fo = P.fwd_off;
    if (plant == 1) {                      // swap blocks 0 and 1 of the first front with two blocks
        bool done = false;
        for (const LevelPlan& lp : P.levels) {
            for (int64_t t = lp.tri_begin; t < lp.tri_begin + lp.tri_count && !done; ++t) {
                if (tt[2 * t + 1] != 0) continue;
                for (int64_t u = t + 1; u < lp.tri_begin + lp.tri_count; ++u)
                    if (tt[2 * u] == tt[2 * t] && tt[2 * u + 1] == 1) {
                        std::swap(tt[2 * t + 1], tt[2 * u + 1]);
                        done = true;
                        break;
                    }
            }
            if (done) break;
        }
        if (!done) return -1;
    } else if (plant == 2) {               // one front's forward partials onto another's
        bool done = false;
        for (const LevelPlan& lp : P.levels) {
            int32_t first = -1;
            for (int32_t js : lp.elim_nodes) {
                if (P.F[js] <= P.S[js]) continue;
                if (first < 0) {
                    first = js;
                } else {
                    fo[js] = fo[first];
                    done = true;
                    break;
                }
            }
            if (done) break;
        }
        if (!done) return -1;
    } else if (plant != 0) {
        return -1;
    }
    int64_t bad = 0, nt = 0;
    // ready flags: one per block of each eliminated large front, disjoint
    {
        std::vector<std::pair<int64_t, int64_t>> iv;
        std::vector<uint8_t> elim(ns, 0);
        for (const LevelPlan& lp : P.levels)
            for (int32_t js : lp.elim_nodes) elim[js] = 1;
        for (int64_t js = 0; js < ns; ++js) {
            if (!elim[js]) continue;
            if (P.tri_off[js] < 0) {
                ++bad;
                continue;
            }
            iv.emplace_back(P.tri_off[js], P.tri_off[js] + (P.S[js] + kNB - 1) / kNB);
        }
        bad += range_faults(iv, P.tri_flags);
    }
    for (const LevelPlan& lp : P.levels) {
        // triangle tasks: each block once, after the block above it
        std::vector<int64_t> first(ns, -1);             // first block-position slot of each front
        std::vector<int64_t> pos;
        for (int32_t js : lp.elim_nodes) {
            first[js] = (int64_t)pos.size();
            pos.resize(pos.size() + (P.S[js] + kNB - 1) / kNB, -1);
        }
        if (lp.tri_begin < 0 || 2 * (lp.tri_begin + lp.tri_count) > (int64_t)tt.size()) {
            ++bad;
            continue;
        }
        for (int64_t t = lp.tri_begin; t < lp.tri_begin + lp.tri_count; ++t) {
            ++nt;
            const int32_t js = tt[2 * t], b = tt[2 * t + 1];
            if (js < 0 || js >= ns || first[js] < 0 || b < 0 || b >= (P.S[js] + kNB - 1) / kNB) {
                ++bad;
                continue;
            }
            int64_t& at = pos[first[js] + b];
            if (at >= 0) ++bad;                                          // listed twice
            at = t;
            if (b > 0 && pos[first[js] + b - 1] < 0) ++bad;              // before the block above it
        }
        for (int64_t v : pos)
            if (v < 0) ++bad;                                            // a block never listed
        // rectangles: one job per front with F > S, of the right sizes, with
        // disjoint partial-sum ranges
        std::vector<int64_t> nrect(ns, 0), nrows(ns, 0);
        std::vector<std::pair<int64_t, int64_t>> riv, fiv;
        for (int64_t j = 0; j < lp.rect.job_count; ++j) {
            const Job& jb = P.jobs[lp.rect.job_begin + j];
            const int32_t js = jb.node;
            if (js < 0 || js >= ns || first[js] < 0) {
                ++bad;
                continue;
            }
            const int64_t f = P.F[js], s = P.S[js];
            const int64_t nrc = (f - s + kRectRows - 1) / kRectRows, ncc = (s + kRectCols - 1) / kRectCols;
            if (f <= s || jb.k_lo != nrc || jb.k_hi != ncc || job_tasks(P, lp.rect, j) != nrc * ncc) ++bad;
            ++nrect[js];
            riv.emplace_back(P.rect_off[js], P.rect_off[js] + nrc * s);
            fiv.emplace_back(fo[js], fo[js] + ncc * (f - s));
        }
        for (int64_t j = 0; j < lp.rect_rows.job_count; ++j) {
            const Job& jb = P.jobs[lp.rect_rows.job_begin + j];
            const int32_t js = jb.node;
            if (js < 0 || js >= ns || first[js] < 0) {
                ++bad;
                continue;
            }
            if (job_tasks(P, lp.rect_rows, j) != (int64_t)P.F[js] - P.S[js]) ++bad;
            ++nrows[js];
        }
        for (int32_t js : lp.elim_nodes) {
            const int64_t want = P.F[js] > P.S[js] ? 1 : 0;
            if (nrect[js] != want || nrows[js] != want) ++bad;
        }
        bad += range_faults(riv, P.rect_entries);
        bad += range_faults(fiv, P.fwd_entries);
    }
    if (tasks) *tasks = nt;
    return bad;
}

int64_t check_schedule(const Plan& P, bool tc, int skip_join) {
    int64_t bad = 0;
    for (const LevelPlan& lp : P.levels) {
        if (lp.elim_nodes.empty()) continue;
        std::map<int32_t, std::vector<SchedOp>> ops;     // per front, in issue order
        int64_t vc[kStreams][kStreams] = {};            // per stream: its vector clock
        int64_t far_done[kStreams], ahead_done[kStreams];
        bool far_open = false, ahead_open = false;
        auto issue = [&](int stream, const Job& j, int kind) {
            ++vc[stream][stream];
            SchedOp o;
            o.stream = stream;
            for (int q = 0; q < kStreams; ++q) o.vc[q] = vc[stream][q];
            o.kind = kind;
            o.k_lo = j.k_lo;
            o.k_hi = j.k_hi;
            if (kind == 0) {                              // panel: columns [k_lo, k_hi), rows to F
                o.c0 = j.k_lo;
                o.c_end = j.k_hi;
                o.r0 = j.k_lo;
                o.r_end = j.r_end;
            } else if (kind == 1) {
                o.c0 = j.c0;
                o.c_end = j.c_end;
                o.r0 = j.c0;
                o.r_end = j.r_end;
            } else {
                o.c0 = 0;
                o.c_end = j.c_end;
                o.r0 = 0;
                o.r_end = j.r_end;
            }
            ops[j.node].push_back(o);
        };
        auto issue_launch = [&](int stream, const Launch& l, int kind) {
            for (int64_t k = 0; k < l.job_count; ++k) issue(stream, P.jobs[l.job_begin + k], kind);
        };
        auto wait = [&](int dst, const int64_t* ev) {       // dst waits for an event
            for (int q = 0; q < kStreams; ++q) vc[dst][q] = std::max(vc[dst][q], ev[q]);
        };
        auto record = [&](int src, int64_t* ev) {
            for (int q = 0; q < kStreams; ++q) ev[q] = vc[src][q];
        };
        auto join = [&]() {
            if (far_open && !(skip_join & 1)) wait(0, far_done);
            far_open = false;
        };
        auto join_ahead = [&]() {
            if (ahead_open && !(skip_join & 2)) wait(0, ahead_done);
            ahead_open = false;
        };
        for (size_t st = 0; st < lp.panel.size(); ++st) {
            issue_launch(0, lp.panel[st], 0);
            const bool has_far = tc ? !lp.far_tc[st].empty() : !lp.far[st].empty();
            if (has_far) wait(1, vc[0]);                 // fork after the step's TRSM
            if ((st + 1) % (kSuperPanel / kNB) == 0) join();
            join_ahead();
            int64_t fork[kStreams];
            record(0, fork);
            for (const Launch& ul : lp.update[st]) issue_launch(0, ul, 1);
            if (!lp.ahead[st].empty()) {
                wait(2, fork);
                for (const Launch& al : lp.ahead[st]) issue_launch(2, al, 1);
                record(2, ahead_done);
                ahead_open = true;
            }
            if (has_far) {
                if (tc)
                    for (const TcLaunch& t : lp.far_tc[st]) issue_launch(1, t.gemm, 1);
                else
                    for (const Launch& fl : lp.far[st]) issue_launch(1, fl, 1);
                record(1, far_done);
                far_open = true;
            }
        }
        join_ahead();
        join();
        if (tc)
            for (const TcLaunch& t : lp.outer_tc) issue_launch(0, t.gemm, 1);
        else
            for (const Launch& ol : lp.outer) issue_launch(0, ol, 1);
        for (int32_t js : lp.elim_nodes) issue(0, Job{js, 0, P.S[js], P.F[js], 0, 0, 0}, 2);
        for (auto& kv : ops) {
            const std::vector<SchedOp>& v = kv.second;
            for (size_t a = 0; a < v.size(); ++a) {
                const SchedOp& A = v[a];
                if (A.kind == 0) {
                    // columns [k0, k0 + nb): K coverage [0, k0) from updates ordered before
                    for (int32_t c = A.c0; c < A.c_end; ++c) {
                        std::vector<std::pair<int32_t, int32_t>> iv;
                        for (const SchedOp& U : v) {
                            if (U.kind != 1 || c < U.c0 || c >= U.c_end) continue;
                            if (!hb(U, A)) {
                                ++bad;
                                continue;
                            }
                            iv.emplace_back(U.k_lo, U.k_hi);
                        }
                        std::sort(iv.begin(), iv.end());
                        int32_t at = 0;
                        bool ok = true;
                        for (const auto& x : iv) {
                            if (x.first != at) ok = false;
                            at = x.second;
                        }
                        if (!ok || at != A.c0) ++bad;
                    }
                } else if (A.kind == 1) {
                    // its K panel columns are final before it
                    for (const SchedOp& Q : v)
                        if (Q.kind == 0 && Q.c0 < A.k_hi && A.k_lo < Q.c_end && !hb(Q, A)) ++bad;
                    // no unordered writer of a common element on the other stream
                    for (size_t b = a + 1; b < v.size(); ++b) {
                        const SchedOp& B = v[b];
                        if (B.kind != 1 || B.stream == A.stream) continue;
                        const bool cols = A.c0 < B.c_end && B.c0 < A.c_end;
                        const bool rows = A.r0 < B.r_end && B.r0 < A.r_end;
                        if (cols && rows && !hb(A, B) && !hb(B, A)) ++bad;
                    }
                } else {
                    for (const SchedOp& U : v)
                        if (U.kind == 1 && U.c0 < A.c_end && !hb(U, A)) ++bad;
                }
            }
        }
    }
    return bad;
}

uint64_t sm_hash_host(const double* a, int64_t n, int threads) {
    const uint64_t* w = reinterpret_cast<const uint64_t*>(a);
    auto part = [w](int64_t i0, int64_t i1) {
        uint64_t acc = 0;
        for (int64_t i = i0; i < i1; ++i) acc += sm_mix(w[i], (uint64_t)i);
        return acc;
    };
    const int64_t per = int64_t(1) << 22;             // below 32 MB one thread is enough
    int nt = (int)std::min<int64_t>(std::max(threads, 1), (n + per - 1) / per);
    if (nt <= 1) return part(0, n);
    std::vector<uint64_t> sums(nt, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([&, t]() { sums[t] = part(n * t / nt, n * (t + 1) / nt); });
    for (auto& th : pool) th.join();
    uint64_t h = 0;
    for (uint64_t v : sums) h += v;
    return h;
}

}  // namespace sprb
