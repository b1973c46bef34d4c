/*
 * spr_b200.h -- C ABI of the B200 numeric phase of SAM's SPR sparse solver.
 *
 * Drop-in entry points (gfortran/ifort-Linux naming: lower case + trailing
 * underscore, every argument by reference, no hidden CHARACTER lengths).
 * SPR_INT is int64_t for libspr_b200.so (the default SPR_I8 build,
 * -fdefault-integer-8, src/SPR/CMakeLists.txt:12-29) and int32_t for
 * libspr_b200_i4.so (BUILD_SPR_INTEGER8=OFF).  The caller owns every array;
 * SM is overwritten by the factor ([D(NEQ) | L(NZEROL)], d on each column's
 * diagonal as in the reference), B by the solution.  IERR, MSPAR(1),
 * MSPAR(26) (NUMNEG) and MSPAR(27) (SUPEQT) and TOL(2:3) follow the
 * reference routines cited below.
 */
#ifndef SPR_B200_H
#define SPR_B200_H

#include <stdint.h>

#ifndef SPR_INT
#define SPR_INT int64_t
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces SPRSOL, src/SPR/sprsol.f:5-52.  IOP<=3 factor, 2<=IOP<=5 forward,
 * IOP>=3 and IOP/=5 back substitution. */
void sprsol_(const SPR_INT* iop, SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm,
             double* b, const SPR_INT* ldb, const SPR_INT* nrhs, double* tol, SPR_INT* iwork,
             double* rwork, const SPR_INT* lpu, SPR_INT* ierr);

/* Replaces SPRFC1, src/SPR/sprfc1.f:5-283 (LDL' factorisation).  MVMULT and
 * MMMULT are the reference's LMVY18/LMMY18 (lmvy18.f:5, lmmy18.f:5); the GPU
 * path always applies the LDL' update they define, so they are not called. */
void sprfc1_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* tol,
             SPR_INT* iwork, double* rwork, const SPR_INT* lpu, SPR_INT* ierr,
             void (*mvmult)(), void (*mmmult)());

/* Replaces SPRFC3, src/SPR/sprfc3.f:5-277 (LDL' factorisation that does not
 * stop on singularity; it is what SPRLAN calls, sprlan.f:814).  TOL(4): on entry
 * TOL(1) is the zero threshold and TOL(4) scales the replacement pivot
 * sign(TOL(1) max(1, |TOL(4) a_jj|), d) (sprfc3.f:1083-1099); a zero diagonal
 * becomes 1 (sprfc3.f:561-572).  DCOR(2,NEQ) receives, per equation, the
 * original pivot (or a negative pivot) and the inserted value.  IERR = -3 with
 * MSPAR(27) = -(number replaced) leaves a complete factor (MSPAR(1) = 5). */
void sprfc3_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* tol,
             SPR_INT* iwork, double* rwork, double* dcor, const SPR_INT* lpu, SPR_INT* ierr,
             void (*mvmult)(), void (*mmmult)());

/* Replaces SPRFC2, src/SPR/sprfc2.f:5-270 (Cholesky C C' factorisation,
 * MSPAR(1) = 6).  A pivot d <= TOL(1)|a_jj| stops it with IERR = -3,
 * MSPAR(27) = the equation, TOL(2) = d and TOL(3) = a_jj (sprfc2.f:1001-1008).
 * MVMULT/MMMULT are CMVY18/CMMY18 (cmvy18.f:5, cmmy18.f:5) and are not called. */
void sprfc2_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* tol,
             SPR_INT* iwork, double* rwork, const SPR_INT* lpu, SPR_INT* ierr,
             void (*mvmult)(), void (*mmmult)());

/* Replaces SPRFC4, src/SPR/sprfc4.f:5-262 (Cholesky C C' with SPRF47's pivot
 * replacement, sprfc4.f:978-1000): TOL(4) and DCOR(2,NEQ) as SPRFC3; a pivot
 * below -TOL(1)|a_jj| stops with IERR = -3, MSPAR(27) = its equation; replaced
 * pivots give IERR = -3, MSPAR(27) = -(number replaced) and a complete factor.
 * MSPAR(1) = 6; MSPAR(26) = 0 as the reference reports it.  MVMULT/MMMULT as
 * SPRFC2 (CMVY18/CMMY18, or null). */
void sprfc4_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* tol,
             SPR_INT* iwork, double* rwork, double* dcor, const SPR_INT* lpu, SPR_INT* ierr,
             void (*mvmult)(), void (*mmmult)());

/* Replaces SPRFS2, src/SPR/sprfs2.f:5-265 (forward sweep C y = b on a C C'
 * factor, MSPAR(1) = 8). */
void sprfs2_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* b,
             const SPR_INT* ldb, const SPR_INT* nrhs, SPR_INT* iwork, double* rwork,
             const SPR_INT* lpu, SPR_INT* ierr);

/* Replaces SPRBS2, src/SPR/sprbs2.f:5-250 (back sweep C' x = y, MSPAR(1) = 8). */
void sprbs2_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* b,
             const SPR_INT* ldb, const SPR_INT* nrhs, double* rwork, const SPR_INT* lpu,
             SPR_INT* ierr);

/* Replaces SPRFS1, src/SPR/sprfs1.f:5-263 (forward reduction + D^-1). */
void sprfs1_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* b,
             const SPR_INT* ldb, const SPR_INT* nrhs, SPR_INT* iwork, double* rwork,
             const SPR_INT* lpu, SPR_INT* ierr);

/* Replaces SPRBS1, src/SPR/sprbs1.f:5-248 (back substitution). */
void sprbs1_(SPR_INT* mspar, SPR_INT* mtrees, SPR_INT* msifa, double* sm, double* b,
             const SPR_INT* ldb, const SPR_INT* nrhs, double* rwork, const SPR_INT* lpu,
             SPR_INT* ierr);

/* ---- device-level API (no reference counterpart: the reference has no
 * device memory; these let a caller keep SM and B resident in HBM) ---- */

/* Builds the execution plan for one SPR structure (arrays as produced by
 * SPRTRS/SPRSMB/SPRPMP, sprtrs.f:5, sprsmb.f:5, sprpmp.f:5).  0 on success. */
int spr_b200_open(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                  void** handle);
void spr_b200_close(void* handle);
/* Runs subsequent work on the given cudaStream_t. */
int spr_b200_set_stream(void* handle, void* stream);
/* Factorises device SM in place (semantics of SPRF11, sprfc1.f:286-713).
 * out[0]=TOL(2) out[1]=TOL(3) out[2]=NUMNEG out[3]=SUPEQT out[4]=LIERR
 * (0, -30 pivot below TOL(1), -35 exact zero diagonal). */
int spr_b200_factor_dev(void* handle, double* d_sm, double tol1, double* out);
/* The same with SPRFC3 semantics (SPRF31, sprfc3.f:372-806): tol = {TOL(1),
 * TOL(4)}, d_dcor = device DCOR(2,NEQ).  out as above; LIERR = -31 and
 * SUPEQT = the number of replaced pivots when any was replaced. */
int spr_b200_factor3_dev(void* handle, double* d_sm, const double* tol, double* d_dcor,
                         double* out);
/* Forward (which=1, SPRFS3 sprfs1.f:266), back (which=2, SPRBS4 sprbs1.f:251)
 * or both (3) on device B (ldb x nrhs, column-major) with device SM. */
int spr_b200_solve_dev(void* handle, const double* d_sm, double* d_b, int64_t ldb,
                       int64_t nrhs, int which);
/* info[0]=RINFO(3) factor flops [1]=solve flops per RHS [2]=front arena bytes
 * [3]=tree levels [4]=last factor ms [5]=last solve ms [6]=launches of the
 * last factorisation [7]=Schur-update launches [8]=Schur-update ms (profile
 * mode) [9]=Schur-update algorithmic flops [10]=launches of the last solve
 * [11]=NZEROL [12]=pivots with |d| < tau |a_jj| that the mixed-mode inertia
 * guard counted in the last factorisation [13]=1 if the guard redid that
 * factorisation in FP64 [14]=trace of the original diagonal (sprfc1.f:483).
 * info must hold 15 doubles. */
int spr_b200_info(void* handle, double* info);
/* Per-supernode negative-pivot counts and first failing column (-1 if none)
 * of the last spr_b200_factor_dev (NSUPER entries each): per-system inertia
 * of a forest of independent systems. */
int spr_b200_sn_stats(void* handle, int32_t* neg, int32_t* fail);
/* Factorisation mode of the device API: 0 = FP64 (default, the drop-in
 * semantics); 1 = mixed precision, the Schur updates of the large fronts as
 * 3xTF32 split products on the tcgen05 tensor cores with FP32 accumulation
 * (FP64 diagonal blocks, TRSM, small fronts and storage); 2 = the same split
 * products through mma.sync (FP64 accumulation every 64 columns).  Pair modes
 * 1 and 2 with spr_b200_refine against the FP64 matrix
 * (spr_b200_build_residual).  Returns -2 for an unknown mode. */
int spr_b200_set_mode(void* handle, int mode);
/* No reference counterpart (the reference has no mixed precision).  Inertia
 * guard of modes 1 and 2: each mixed factorisation first keeps a copy of the
 * assembled device SM (one extra SM-sized buffer, allocated once); when it
 * meets a pivot with |d| < tau |a_jj| (a_jj the original diagonal) or a
 * failed pivot test, its sign or the test may depend on the TF32 rounding,
 * so the factorisation is redone in FP64 from that copy and NUMNEG, IERR and
 * TOL are the FP64 ones (the pivot rule of SPRF17, sprfc1.f:1272-1283).
 * Default tau = 1e-3; tau = 0 switches the guard and the copy off. */
int spr_b200_set_inertia_guard(void* handle, double tau);
/* No reference counterpart.  Watchdog of the kernels that wait on device
 * flags: the tensor-core update kernel's mbarrier waits and the solves'
 * block-ready flags each give up after wait_ns nanoseconds (default 2e9;
 * 1e6 .. 6e10 accepted); the kernel then returns (the tensor-core one after
 * freeing its tensor memory) and the factorisation or solve returns -4.
 * drop != 0 is a test switch: the first CTA of each tensor-core launch skips
 * its first operand load and one task of each solve triangle launch never
 * reports its block, so that waits run out.  Returns -2 for a limit outside
 * the range. */
int spr_b200_set_watchdog(void* handle, double wait_ns, int drop);
/* No reference counterpart.  One system split across GPUs (one process and
 * one handle per GPU, the same structure on all; orchestrated by
 * sam_lib_b200/split.py).  spr_b200_set_skip: supernodes with mask[js] != 0
 * (NSUPER bytes) are left alone by spr_b200_factor_dev and spr_b200_solve_dev;
 * NULL clears the mask.  spr_b200_set_exchange: for the following
 * factorisations, node fo_node[k]'s update block ((F-S) x (F-S) doubles,
 * column-major, leading dimension F-S) is copied to the device buffer
 * fo_buf[k] right after that node's tree level, and fi_buf[k] is copied into
 * node fi_node[k]'s block right before its parent's level; for the following
 * forward sweeps the same with the update vectors ((F-S) x nrhs doubles, nrhs
 * <= 16), vo_* and vi_*.  Copies run on the handle's stream.  -2 for a bad
 * node or buffer. */
int spr_b200_set_skip(void* handle, const uint8_t* mask);
int spr_b200_set_exchange(void* handle, int64_t nfo, const int32_t* fo_node, double* const* fo_buf,
                          int64_t nfi, const int32_t* fi_node, double* const* fi_buf, int64_t nvo,
                          const int32_t* vo_node, double* const* vo_buf, int64_t nvi,
                          const int32_t* vi_node, double* const* vi_buf);
/* Residual operator for refinement: compacts the FP64 matrix held in an
 * assembled (not yet factored) device SM into a CSR (the product SPRPRQ forms
 * from the packed pattern, sprprm.f:243-325). */
int spr_b200_build_residual(void* handle, const double* d_sm_assembled);
/* Iterative refinement on a factored device SM: x = solve(b); while the
 * normwise backward error max|r|/(||K||inf max|x| + max|b|) > tol and fewer
 * than maxit corrections: x += solve(b - K x).  out[0]=corrections
 * out[1]=backward error out[2]=solve ms.  b, x: ld x nrhs, device. */
int spr_b200_refine(void* handle, const double* d_sm, const double* d_b, double* d_x, int64_t ld,
                    int64_t nrhs, double tol, int maxit, double* out);
/* Profile mode only: last factorisation's time by phase, out[0..8] = pre-pass,
 * small fronts, extend-add, diagonal blocks, panel TRSM, in-panel/trailing
 * updates, K = S update, write-back, end; last solve's, out[9..19] =
 * forward: small fronts, gather, blocks, rectangles, finish;
 * back: small fronts, gather, rectangles, blocks, (unused), finish (ms).  out holds 20 doubles. */
int spr_b200_phase_ms(void* handle, double* out);
/* No reference counterpart.  Autotuner of the mixed-precision factorisation:
 * it times candidate choices (which Schur-update launches run on the tensor
 * cores, by a minimum of algorithmic flops; how many SMs the side-stream
 * launches may take), each on a copy of the assembled device SM (one extra
 * SM-sized buffer is allocated for the duration), and keeps the fastest for
 * later factorisations.  out[0] = chosen minimum flops, out[1] = chosen
 * quarters of the SMs, out[2] = its factor ms, out[3] = the default's,
 * out[4] = candidates tried. */
int spr_b200_autotune(void* handle, const double* d_sm_assembled, double* out);
/* No reference counterpart.  Tile autotuner of the small FP64 Schur updates
 * (those with fewer than 256 rows): factors a copy of d_sm_assembled with
 * 64x64 and with 32x32 update tiles and keeps the faster.  out (3 doubles):
 * the tile chosen, factor ms with 64, factor ms with 32. */
/* No reference counterpart.  Self-test of the pivot reciprocal of the
 * diagonal-block kernels (a hardware approximation refined by two
 * Newton-Raphson steps): out[2i] = it for x[i], out[2i+1] = the IEEE quotient
 * 1.0 / x[i], computed on the device (host arrays, n values). */
int spr_b200_recip_check(const double* x, int64_t n, double* out);
int spr_b200_autotune_tiles(void* handle, const double* d_sm_assembled, double* out);
/* Sets that tile explicitly (64 or 32). */
int spr_b200_set_small_tile(void* handle, int tile);
/* Mixed mode: out[0] = algorithmic flops of the Schur updates that run on the
 * tensor cores (trailing columns beyond the next super-panel, K = S updates),
 * out[1] = their split + tensor-core time in the last profiled factor (ms). */
int spr_b200_tc_stats(void* handle, double* out);
/* Profile mode: CUDA events around every Schur-update launch. */
int spr_b200_set_profile(void* handle, int on);
/* Host-only plan build + self-check (no GPU needed).  out (13 doubles):
 * [0] build status [1] NSUPER [2] tree levels [3] front arena doubles
 * [4] buffers outside the arena plus relative-index (SPRF12 LINDEX) and
 * contribution-list entries out of range or not used exactly once
 * [5] overlapping live buffers [6] RINFO(3)
 * [7] solve flops per RHS [8] small fronts [9] large fronts [10] jobs
 * [11] columns whose FP64 Schur-update K ranges do not tile the earlier
 * panels (all S columns, for update columns) exactly once [12] the same for
 * the mixed mode's launch lists. */
int spr_b200_plan_check(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                        double* out);
/* Host-only race check of the factorisation's three-stream launch schedule (no
 * GPU needed): happens-before of panels, panel-chain, look-ahead, far and K = S
 * updates and the write-back.  out (6 doubles): [0] ordering violations of the
 * FP64 schedule [1] of the schedule with tensor-core far and K = S updates
 * [2] of the FP64 schedule without its side-stream joins (a self-test; > 0
 * when [3] > 0) [3] far launches [4] of the FP64 schedule without its
 * look-ahead joins (> 0 when [5] > 0) [5] look-ahead launches. */
int spr_b200_schedule_check(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                            double* out);
/* No reference counterpart.  Host-only self-check of the solves' plan (no GPU
 * needed): each eliminated large front's 64-row triangle blocks are tasks of
 * its level's dataflow launch, once each and after the block above, with
 * disjoint ready flags; each front with F > S has one rectangle job and one
 * forward-rows job of the right sizes, with disjoint partial-sum ranges.
 * out (5 doubles): [0] rc [1] violations [2] triangle tasks checked [3] and
 * [4] violations with a planted mistake (two blocks of a front swapped; one
 * front's forward partials moved onto another's): > 0, or -1 where no front
 * of the structure admits the mistake. */
int spr_b200_solve_plan_check(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                              double* out);
/* Host element assembly into LNZ, the SPRADM/SPRAD2 main add
 * (src/SPR/spradm.f:818-859) for systems without constraint equations:
 * SM(NEQ+K) += EM(I,J), J=1..NEDOF, I<=J, elements in order (bit-exact with
 * SPRADM).  EM of element e = em_scale[e]*em, or the e-th matrix of em when
 * em_scale is NULL.  MEQN as renumbered by SPRTRS/SPREQN (sprtrs.f:3762).
 * Returns 0, or -3 on a DOF count or pattern mismatch. */
int spr_b200_assemble(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                      const SPR_INT* meqn, const SPR_INT* madof, const SPR_INT* mpmnpc,
                      const SPR_INT* mmnpc, SPR_INT nel, SPR_INT nedof, const double* em,
                      const double* em_scale, double* sm);
/* Replaces SPRADM (src/SPR/spradm.f:5) called once per element in order,
 * constraint equations included: SPRAD2's free-DOF add and its weighted
 * additions for slave DOFs (TTCC master coefficients) and prescribed DOFs
 * (TTCC constant terms into SV), spradm.f:818-1002, bit-exact.  MPMCEQ
 * (nceq+1), MMCEQ, TTCC as SAM holds them; nsv as SPRADM's NSV (0: SM only,
 * 1: SM and SV, -1: SV only; SV has NEQ entries and is accumulated into).
 * Returns 0, -2 (|nsv| > 1, the multi-load-case SV, is not supported) or -3. */
int spr_b200_assemble_ceq(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                          const SPR_INT* meqn, const SPR_INT* madof, const SPR_INT* mpmnpc,
                          const SPR_INT* mmnpc, const SPR_INT* mpmceq, const SPR_INT* mmceq,
                          const double* ttcc, SPR_INT nceq, SPR_INT nel, SPR_INT nedof,
                          const double* em, const double* em_scale, SPR_INT nsv, double* sm,
                          double* sv);
/* No counterpart in the reference (SPR never touches device memory).
 * LDL' of one dense symmetric front on the device, in place, for callers that
 * must not allocate device memory (an application allocator owns it all, or
 * an allocation would stall a time-critical loop): d_a (n x n, column-major,
 * leading dimension lda % 4 == 0, 32-byte aligned, lower triangle used) is
 * overwritten by L below the diagonal and d on it; d_d (n) receives d.  All
 * scratch lives in one 5 MiB file-scope __device__ array, so n <= 8192
 * (else -3); calls that overlap on the GPU race on that array; the first call
 * on a device resolves its address and should precede any stream capture.
 * Pivot test, inertia and TOL(2) as SPRF17 (sprfc1.f:1272-1294).
 * out[0]=NUMNEG out[1]=first failing column (1-based, 0 if none)
 * out[2]=that pivot out[3]=its original a_jj out[4]=max(a_jj/d_j).
 * Returns 0, -2 (shape/alignment), -3 (too large) or -4 (CUDA error). */
int spr_b200_dense_ldlt_noalloc(double* d_a, int64_t n, int64_t lda, double tol1, double* d_d,
                                void* stream, double* out);
/* ---- element-level device operations (no reference counterpart for the
 * gradient; the assembly is SPRADM's main add) ---- */
/* Builds the gather plan of the SPRADM main add (spradm.f:818-859) and the
 * element equation map for one structure and SAM element topology (MEQN,
 * MADOF, MPMNPC, MMNPC as SPRADM takes them; every element has nedof <= 32
 * DOFs, nel < 2^22).  0, -2 (limits), -3 (DOF count or pattern mismatch). */
int spr_b200_elem_open(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                       const SPR_INT* meqn, const SPR_INT* madof, const SPR_INT* mpmnpc,
                       const SPR_INT* mmnpc, SPR_INT nel, SPR_INT nedof, void** handle);
/* The same with constraint equations (MPMCEQ, MMCEQ as SAM holds them,
 * nceq = MPAR(7)): the plan also holds SPRAD2's weighted additions and the
 * SV gather of the prescribed values. */
int spr_b200_elem_open_ceq(const SPR_INT* mspar, const SPR_INT* mtrees, const SPR_INT* msifa,
                           const SPR_INT* meqn, const SPR_INT* madof, const SPR_INT* mpmnpc,
                           const SPR_INT* mmnpc, const SPR_INT* mpmceq, const SPR_INT* mmceq,
                           SPR_INT nceq, SPR_INT nel, SPR_INT nedof, void** handle);
void spr_b200_elem_close(void* handle);
/* Device SM = 0 then the SPRADM main add of every element: EM_e =
 * d_scale[e]*d_em (one nedof x nedof column-major matrix) or, with d_scale
 * NULL, the e-th matrix of d_em.  Bit-exact with spr_b200_assemble. */
int spr_b200_elem_assemble(void* handle, double* d_sm, const double* d_em, const double* d_scale,
                           void* stream);
/* SPRADM with constraint equations on the device (a handle from
 * spr_b200_elem_open_ceq): device SM = 0 and/or SV = 0 (NEQ), then every
 * element's additions in SPRADM's order and rounding with the coefficients
 * of the device array d_ttcc; bit-exact with spr_b200_assemble_ceq.  d_sm or
 * d_sv NULL skips that part (NSV = -1 or 0).  -2 when d_ttcc is NULL and the
 * plan has weighted additions. */
int spr_b200_elem_assemble_ceq(void* handle, double* d_sm, double* d_sv, const double* d_em,
                               const double* d_scale, const double* d_ttcc, void* stream);
/* No reference counterpart (SAM ships no element routines): the 24x24
 * stiffness of every element, an 8-node isoparametric hexahedron with
 * 2x2x2 Gauss integration, isotropic with Young's modulus d_E[e] and
 * Poisson's ratio nu, from the node coordinates d_xyz (NANOD x 3, row per
 * SAM node number - 1; corners in the order (0,0,0) (1,0,0) (1,1,0) (0,1,0)
 * (0,0,1) (1,0,1) (1,1,1) (0,1,1) of the element's MMNPC).  d_em receives
 * NEL column-major matrices with node-major DOFs (3a + x/y/z), the layout
 * spr_b200_elem_assemble reads.  -2 unless every element has 8 nodes of 3
 * DOFs. */
int spr_b200_elem_hex8(void* handle, const double* d_xyz, const double* d_E, double nu, double* d_em,
                       void* stream);
/* Adjoint element gradient: d_grad[e] = -sum_q lam_q,e^T dK_e u_q,e with
 * dK_e = d_dscale[e]*d_em, or the e-th matrix of d_em when d_dscale is NULL;
 * u, lam: ld x nrhs device arrays in equation order (constrained DOFs are
 * skipped).  With lam solving K lam = dL/du this is dL/dtheta_e. */
int spr_b200_elem_grad(void* handle, const double* d_u, const double* d_lam, int64_t ld, int64_t nrhs,
                       const double* d_em, const double* d_dscale, double* d_grad, void* stream);
/* No reference counterpart.  Timing of the last factorisation through the
 * Fortran entry points on a page-locked SM (copies overlapped with the
 * factorisation): out[0] = ms of upload before the first level could start,
 * out[1] = factorisation ms, out[2] = ms of download after its end (3 doubles). */
int spr_b200_copy_stats(double* out);
/* No reference counterpart.  The number of device contexts the Fortran entry
 * points hold (one per MSPAR/MTREES/MSIFA triple they were called with). */
int spr_b200_contexts(void);
/* Frees every device context cached by the Fortran entry points. */
void spr_b200_release_all(void);

#ifdef __cplusplus
}
#endif
#endif /* SPR_B200_H */
