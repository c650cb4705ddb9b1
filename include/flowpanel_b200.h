/*
 * flowpanel_b200.h — C ABI of the B200 (sm_100a) panel-method hot path.
 *
 * Drop-in boundary for FLOWPanel.jl's dense solve path: a Julia solver object
 * calls these entry points through `ccall` (the bindings are in
 * flowpanel.jl_b200/julia/FLOWPanelB200.jl); the Python host mirror in
 * flowpanel.jl_b200/ calls them through ctypes.
 *
 * Conventions (Julia's column-major layouts, passed zero-copy):
 *   nodes       3 x nnodes  double   (x0,y0,z0,x1,...)
 *   panels      CSR: panel_offsets[npanels+1], panel_nodes[] 0-based node
 *               indices, 3 or 4 nodes per panel (planar)
 *   cps/normals 3 x npanels double (control points and unit normals)
 *   shedding    6 x nsh int32: (pi, nia, nib, pj, nja, njb), 0-based panel
 *               index and panel-local node indices, pj == -1 for no lower side
 *   Das/Dbs     3 x nsh double, unit vectors
 *   G           N x N column-major (column j = unit-strength influence of
 *               panel j on every control point)
 * All host buffers belong to the caller and are read (or, for outputs,
 * written) during the call only. Device memory belongs to the context.
 * Every entry point returns FP_OK (0) or an FP_E* status; fp_last_error()
 * gives the text. Calls on one context are serialised by the caller; separate
 * contexts may run concurrently.
 */
#ifndef FLOWPANEL_B200_H
#define FLOWPANEL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FP_OK 0
#define FP_EINVAL 1      /* bad argument (shape, non-unit direction, ...) */
#define FP_ESINGULAR 2   /* zero pivot in the factorisation */
#define FP_ENOCONV 3     /* iterative solver did not reach its tolerance */
#define FP_ECUDA 4       /* CUDA runtime error */
#define FP_ETIMEOUT 5    /* a bounded device-side wait ran out */
#define FP_ESTATE 6      /* call out of order (e.g. solve before factor) */

/* element kinds */
#define FP_ELEMENT_SOURCE 0      /* NonLiftingBody{ConstantSource} */
#define FP_ELEMENT_VORTEXRING 1  /* RigidWakeBody / MultiBody {VortexRing}; NonLiftingBody{ConstantDoublet}
                                    (the same element without a wake) */
#define FP_ELEMENT_SOURCE_DOUBLET 2  /* NonLiftingBody{Union{ConstantSource, ConstantDoublet}}: strengths N x 2
                                        (sources, then doublets); fp_uind and fp_phi only */

/* precision forms */
#define FP_PREC_FP64 0   /* FP64 assembly + FP64 LU (the plain form) */
#define FP_PREC_MIXED 1  /* FP32 factors with a static row order (no pivot search; 3xTF32 tensor-core
                            update) + FP64 refinement, GMRES-IR behind it; a zero pivot, or refinement
                            that fails, falls back to FP_PREC_MIXED_GEPP */
#define FP_PREC_MIXED_GEPP 2  /* FP32 factors pivoted as the FP64 form (partial pivoting inside each
                                 64-row diagonal block) + FP64 refinement */
#define FP_PREC_BF16 3   /* the largest meshes: the factorisation starts from the BF16-rounded AIC and
                            its trailing update multiplies BF16 operands (tcgen05 kind::f16) with FP32
                            accumulation, static row order; refinement hands over to GMRES-IR with
                            FP64 residuals on the FP64 AIC, which recovers ir_tol */

/* solvers */
#define FP_SOLVER_LU 0     /* solve_ludiv! / solve_backslash! */
#define FP_SOLVER_GMRES 1  /* solve_gmres! (restarted GMRES on the FP64 AIC) */

typedef struct fp_ctx fp_ctx;

typedef struct fp_solve_opts {
  int solver;          /* FP_SOLVER_* */
  int precision;       /* FP_PREC_*; for FP_SOLVER_LU the factor precision */
  double ir_tol;       /* mixed: stop refining when ||b-Ax||_2 <= ir_tol*||b||_2 (<=0: 1e-12) */
  int ir_maxiter;      /* mixed: refinement steps before GMRES-IR takes over (<=0: 10) */
  int gmres_memory;    /* restart length (<=0: 50) */
  double gmres_atol;   /* <0: sqrt(eps) */
  double gmres_rtol;   /* <0: sqrt(eps) */
  int gmres_itmax;     /* <=0: 2N */
  int gmres_restart;   /* 0: one Arnoldi process whose basis grows past gmres_memory (Krylov.jl 0.9's
                          gmres with restart = false, the reference's call); 1: GMRES(gmres_memory) */
} fp_solve_opts;

typedef struct fp_stats {
  double ms_assemble;  /* device time of the last fp_assemble */
  double ms_factor;    /* device time of the last fp_factor */
  double ms_solve;     /* device time of the last fp_solve */
  int ir_iters;        /* refinement steps of the last mixed solve */
  int gmres_iters;     /* GMRES iterations of the last solve (all RHS) */
  int used_gmres;      /* 1 if GMRES(-IR) produced the last solution */
  int gepp_certified;  /* 1 if every pivot equals LAPACK dgetrf's choice */
  double max_abs_L;    /* largest |L| entry below the diagonal blocks */
  double rel_residual; /* max over RHS of ||b-Ax||_2/||b||_2 (FP64) */
} fp_stats;

/* Context: one CUDA device, one stream. Replaces the per-solve allocations of
 * src/FLOWPanel_liftingbody.jl:191-199 (G = zeros(T, N, N), Gamma = zeros). */
int fp_ctx_create(int device, fp_ctx** ctx);
int fp_ctx_destroy(fp_ctx* ctx);
const char* fp_last_error(const fp_ctx* ctx);
/* 1 if the library was built with the sm_100a kernels and a device is usable */
int fp_device_count(void);

/* Geometry of the body (or the concatenated bodies of a MultiBody, in body
 * order, src/FLOWPanel_multibody.jl:502-530). cps/normals are the ones
 * _calc_controlpoints!/_calc_normals! produce (src/FLOWPanel_abstractbody.jl:635-755);
 * NULL asks the library to compute them with off = cp_offset[i] * l = 1
 * (pass cp_offset = NULL for the default 1e-14). */
int fp_set_geometry(fp_ctx* ctx, const double* nodes, int64_t nnodes,
                    const int32_t* panel_offsets, const int32_t* panel_nodes,
                    int64_t npanels, const double* cps, const double* normals,
                    const double* cp_offset);

/* Kutta wake: the shedding matrix and the semi-infinite directions
 * (src/FLOWPanel_liftingbody.jl:508-567, inputs of _G_Uvortexring!).
 * Non-unit directions -> FP_EINVAL (src/FLOWPanel_elements.jl:495-498). */
int fp_set_wake(fp_ctx* ctx, const int32_t* shedding, int64_t nsh, const double* Das,
                const double* Dbs);

/* Dense AIC assembly G = _G_U!(...): constant source
 * (src/FLOWPanel_nonliftingbody.jl:141-186) or vortex rings plus the Kutta wake
 * columns (src/FLOWPanel_liftingbody.jl:455-572). Always FP64 in HBM; with
 * FP_PREC_MIXED an FP32 copy for the factorisation is written by the same pass. */
int fp_assemble(fp_ctx* ctx, int element, double kerneloffset, double kernelcutoff,
                int precision);

/* Copy the assembled FP64 AIC to the host (N x N column-major). */
int fp_get_aic(fp_ctx* ctx, double* G);

/* Right-hand sides calc_bc_noflowthrough!: RHS_i = -Uinf_i . n_i
 * (src/FLOWPanel_linearsolver.jl:297-312). Uinfs is 3 x N x k. */
int fp_set_rhs(fp_ctx* ctx, const double* Uinfs, int64_t k);

/* LU factorisation calc_Alu / LA.lu! (src/FLOWPanel_linearsolver.jl:173-234). */
int fp_factor(fp_ctx* ctx, int precision);

/* Solve for the k right-hand sides set by fp_set_rhs: solve_ludiv! /
 * solve_backslash! / solve_gmres! (src/FLOWPanel_linearsolver.jl:24-157).
 * x is N x k (column-major) on the host. opts may be NULL (LU, FP64). */
int fp_solve(fp_ctx* ctx, double* x, int64_t k, const fp_solve_opts* opts, fp_stats* stats);

/* Solve A X = B in place with the FP64 LU factors of the last
 * fp_factor(ctx, FP_PREC_FP64), on caller-owned DEVICE memory, allocating no
 * device memory. No counterpart in the reference (its solves allocate their
 * results); it is for callers that cannot let a library allocate during a
 * solve: a host program whose own pool or arena holds the device memory (a
 * Julia session with CUDA.jl's pool, a fixed-budget service), or a loop of
 * re-solves where a cudaMalloc could synchronise the device or fail.
 * B: n x k column-major on ctx's device, leading dimension ldb >= n; it is
 * read and written on ctx's stream, which does not wait for the caller's
 * streams, so finish writing B first. The call returns when the solve is done.
 * Limit: n <= 65536 (FP_EINVAL beyond): the triangular solves keep their
 * ready flags and ticket counter in a fixed static device array (4 KiB per
 * device); each sweep zeroes them itself, so nothing needs initialising.
 * Every call resolves that array's address with cudaGetSymbolAddress; the
 * first call on a device can load the library's device code onto it, so make
 * that call before any stream capture. FP64 factors whose block-local pivots
 * are not certified (fp_stats.gepp_certified == 0) are refused with
 * FP_ESTATE: fp_solve refines those. Calls that overlap in time on
 * one device (several host threads, several contexts) share the array and
 * race, giving wrong results or FP_ETIMEOUT: serialise them. */
int fp_lu_solve_noalloc(fp_ctx* ctx, double* B, int64_t ldb, int64_t k);

/* End-to-end solve(body, Uinfs, Das, Dbs; solver) for a body already given by
 * fp_set_geometry/fp_set_wake: assemble + RHS + factor + solve
 * (src/FLOWPanel_liftingbody.jl:172-216, src/FLOWPanel_multibody.jl:312-364,
 * src/FLOWPanel_nonliftingbody.jl:93-130). */
int fp_solve_body(fp_ctx* ctx, int element, double kerneloffset, double kernelcutoff,
                  const double* Uinfs, int64_t k, const fp_solve_opts* opts, double* x,
                  fp_stats* stats);

/* One body of a batch: the arguments of fp_set_geometry, fp_set_wake and
 * fp_solve_body for one body (host arrays, read during the call only; cps and
 * normals may be NULL; shedding/Das/Dbs unused for FP_ELEMENT_SOURCE). */
typedef struct fp_body_desc {
  const double* nodes;          /* 3 x nnodes */
  int64_t nnodes;
  const int32_t* panel_offsets; /* npanels + 1 */
  const int32_t* panel_nodes;
  int64_t npanels;
  const double* cps;            /* 3 x npanels or NULL */
  const double* normals;        /* 3 x npanels or NULL */
  const int32_t* shedding;      /* 6 x nsh */
  int64_t nsh;
  const double* Das;            /* 3 x nsh */
  const double* Dbs;            /* 3 x nsh */
  const double* Uinfs;          /* 3 x npanels */
  double* x;                    /* out: npanels strengths */
} fp_body_desc;

/* Batched solves of many bodies of uneven panel counts (the batching form;
 * no counterpart in the reference, whose solve takes one body at a time).
 * A batch owns nslots contexts on one device; fp_batch_solve assembles,
 * factors and solves every body with opts (as fp_solve_body does, so each
 * result equals a single solve's), nslots bodies at a time, largest first,
 * one host thread per slot. stats (nbody entries) may be NULL. On failure the
 * status of the first failing body is returned and fp_batch_last_error names
 * it; the other bodies are still solved. */
typedef struct fp_batch fp_batch;
int fp_batch_create(int device, int nslots, fp_batch** out);
int fp_batch_destroy(fp_batch* batch);
const char* fp_batch_last_error(fp_batch* batch);
int fp_batch_solve(fp_batch* batch, int element, double kerneloffset, double kernelcutoff, int64_t nbody,
                   const fp_body_desc* bodies, const fp_solve_opts* opts, fp_stats* stats);

/* Induced velocity Uind! of the solved body on m targets, accumulated into
 * out (3 x m): vortex rings + wake horseshoes with (Gamma_pi, Gamma_pj)
 * (src/FLOWPanel_liftingbody.jl:576-661), constant sources
 * (src/FLOWPanel_nonliftingbody.jl:188-218), or sources then doublets
 * (FP_ELEMENT_SOURCE_DOUBLET, :719-761), with the body's kerneloffset and
 * kernelcutoff. precision FP_PREC_MIXED evaluates in FP32 (off-body probes). */
int fp_uind(fp_ctx* ctx, int element, const double* strengths, const double* targets,
            int64_t m, double* out, int precision, double kerneloffset, double kernelcutoff);

/* Least-squares solve of a watertight vortex-ring body, the
 * RigidWakeBody{VortexRing, 2} / MultiBody{VortexRing, 2} method
 * (src/FLOWPanel_liftingbody.jl:236-447, src/FLOWPanel_multibody.jl:373-617):
 * assembles G (with the wake set by fp_set_wake), moves the npres prescribed
 * strengths (0-based el_index, values el_value; sorted here, distinct) to the
 * right-hand side, solves the normal equations Gred^T Gred Gamma = Gred^T r
 * in FP64 with LU (solve_ludiv!, the default solver) and writes Gamma (N) with
 * the prescribed values in place (set_solution). Leaves no usable factors of
 * G (call fp_factor again before fp_solve). */
int fp_solve_ls(fp_ctx* ctx, double kerneloffset, double kernelcutoff, const double* Uinfs, int64_t npres,
                const int64_t* el_index, const double* el_value, double* x, fp_stats* stats);

/* Potential phi! of the solved body on m targets, accumulated into out (m):
 * constant sources (src/FLOWPanel_nonliftingbody.jl:221-250), constant
 * doublets (:388-420, FP_ELEMENT_VORTEXRING without a wake), both
 * (FP_ELEMENT_SOURCE_DOUBLET, :763-815, strengths N x 2), or vortex rings with
 * the wake's semi-infinite doublets, (da, db) on the upper TE nodes with the
 * upper panel's strength and (db, da) on the lower's
 * (src/FLOWPanel_liftingbody.jl:664-742; elements :152-241, 751-847,
 * 959-1244). FP64. FP_EINVAL with the reference's message when a shedding
 * edge's da and db are opposite or orthogonal (:1129-1132). */
int fp_phi(fp_ctx* ctx, int element, const double* strengths, const double* targets, int64_t m,
           double* out, double kerneloffset);

/* Surface velocity from the gradient of the doublet strength of a solved body
 * with triangular panels, added to out (N x 3):
 *   FP_UGRADMU_COMBINED  calcfield_Ugradmu! (src/FLOWPanel_postprocess.jl:825-941):
 *       the cell scheme, except on cells with a free edge or a neighbour whose
 *       normal is more than anglecrit degrees off, which take the node scheme
 *       (with the cell values on the trailing-edge cells pi, pi+1, pj, pj-1
 *       when force_cellTE); out_cell / out_node (N x 3, may be NULL) receive
 *       the two schemes' fields;
 *   FP_UGRADMU_CELL      calcfield_Ugradmu_cell! (:139-540): Green-Gauss with
 *       the inverse-distance face value, the face terms of the shedding rows'
 *       pi/pj cells added back, rows whose norm reaches maxgrad zeroed;
 *   FP_UGRADMU_NODE      calcfield_Ugradmu_node! (:622-748, sharpTE = false):
 *       out is overwritten with -1/2 the gradient of the area-weighted nodal
 *       values.
 * strength: the N doublet strengths (Gammai column); cp_offset: per panel
 * CPoffset (its sign flips the field, NULL = all positive). Neighbours are the
 * panels sharing an edge (the wake's shedding rows from fp_set_wake).
 * FP_EINVAL for a non-triangular panel or an edge of more than two panels.
 * FP64; device time: fp_last_kernel_ms(FP_STAGE_POST). */
#define FP_UGRADMU_COMBINED 0
#define FP_UGRADMU_CELL 1
#define FP_UGRADMU_NODE 2
int fp_ugradmu(fp_ctx* ctx, int scheme, const double* strength, const double* cp_offset, double anglecrit,
               int force_cellTE, double maxgrad, double* out, double* out_cell, double* out_node);

/* fp_ugradmu with the schemes' remaining options (fp_ugradmu is this call with
 * sharpTE = 0 and no smoothing):
 *   sharpTE (node and combined schemes; calcfield_Ugradmu_node!'s sharpTE,
 *       src/FLOWPanel_postprocess.jl:698-742): the trailing-edge cells take,
 *       at the trailing-edge nodes (the nodes of each shedding row's upper
 *       edge), the area-weighted nodal value over their own side's cells only:
 *       upper cells pi, pi+1, lower cells pj, pj-1, the lower side last;
 *   smooth_cells / nsmooth / smooth_pass (cell scheme; smoothRows and
 *       smoothPass, :499-526): after all gradients, smooth_pass times, each
 *       listed cell in list order takes the mean of its edge neighbours'
 *       current values; the maxgrad cut follows the smoothing. The list is
 *       the cells of smoothRows, in the reference's row-then-span order.
 * FP_EINVAL for a cell index outside 0..N-1 or negative counts. */
int fp_ugradmu_ex(fp_ctx* ctx, int scheme, const double* strength, const double* cp_offset, double anglecrit,
                  int force_cellTE, double maxgrad, int sharpTE, const int32_t* smooth_cells, int64_t nsmooth,
                  int smooth_pass, double* out, double* out_cell, double* out_node);

/* calcfield_Cp! (src/FLOWPanel_postprocess.jl:1059-1112): out (N) +=
 * 1 - (|U|/Uref)^2 for the velocities Us (N x 3), then, with correct_kutta,
 * the average over (pi, pi+1, pj, pj-1) of each shedding row in row order. */
int fp_calcfield_cp(fp_ctx* ctx, const double* Us, double Uref, int correct_kutta, double* out);

/* calcfield_F! (src/FLOWPanel_postprocess.jl:1199-1307): out (N x 3) +=
 * -Cp (rho Uinf^2 / 2) A n with the normals flipped by sign(cp_offset), then,
 * with correct_kutta, the forces of each shedding row's cells overwritten
 * from their average Cp. */
int fp_calcfield_f(fp_ctx* ctx, const double* Cps, const double* cp_offset, double Uinf, double rho,
                   int correct_kutta, double* out);

/* calcfield_LDS! (src/FLOWPanel_postprocess.jl:1615-1652): out (3 x 3,
 * column-major: lift, drag, sideslip vectors) from the sum of Fs (N x 3) added
 * to out's third column, projected on the unit vectors Lhat, Dhat, Shat
 * (FP_EINVAL with the reference's message when one is not unitary). */
int fp_calcfield_lds(fp_ctx* ctx, const double* Fs, const double* Lhat, const double* Dhat, const double* Shat,
                     double* out);

/* The surface loads of a solved body in one pass on the device, the sequence
 * of examples/sweptwing_solverbenchmark.jl:14-66: U = Uinfs + Uind at the
 * control points (calcfield_U), + the combined grad(mu) velocity when ugradmu
 * (anglecrit 30, force_cellTE), Cp with Uref and the Kutta average when
 * correct_kutta, F with Uinf = Uref and rho, and L/D/S. Outputs: U (N x 3,
 * may be NULL), Cp (N), F (N x 3), LDS (3 x 3 column-major). Device time
 * (induced velocity to L/D/S): fp_last_kernel_ms(FP_STAGE_POST). */
int fp_surface_loads(fp_ctx* ctx, int element, const double* strengths, const double* Uinfs,
                     const double* cp_offset, double kerneloffset, double kernelcutoff, int ugradmu,
                     double Uref, double rho, const double* Lhat, const double* Dhat, const double* Shat,
                     int correct_kutta, double* U, double* Cp, double* F, double* LDS);

/* Adjoint of the linear solve: A^T lambda = ybar with the saved factors (the
 * reverse rule of IAD.implicit_linear at src/FLOWPanel_linearsolver.jl:73:
 * lambda = A^-T ybar, Abar = -lambda x^T, bbar = lambda). ybar/lambda N x k on
 * the host. With FP64 factors one transposed LU solve; with the FP32 factors
 * of FP_PREC_MIXED, iterative refinement against the FP64 AIC to a relative
 * residual of 1e-12 (FP_ENOCONV if it stalls). The solution also stays on the
 * device for fp_assembly_vjp. Device time: fp_last_kernel_ms(FP_STAGE_ADJOINT). */
int fp_adjoint_solve(fp_ctx* ctx, const double* ybar, int64_t k, double* lambda);

/* Reverse mode of the vortex-ring assembly (the pullback that ForwardDiff
 * through _G_Uvortexring! and calc_bc_noflowthrough! gives the reference's
 * ImplicitAD path, src/FLOWPanel_liftingbody.jl:455-572,
 * src/FLOWPanel_linearsolver.jl:297-312): the gradient of
 * lambda^T (b - A Gamma), b_i = -Uinf_i . n_i, with respect to the ring and
 * wake-node coordinates (dnodes, 3 x nnodes), the control points (dcps, 3 x N),
 * the normals (dnormals, 3 x N), the freestream at each control point
 * (dUinfs, 3 x N) and the wake directions (dDas, dDbs, 3 x nsh). With
 * lambda = A^-T dF/dGamma (fp_adjoint_solve) this is the total derivative of
 * F through the solve. lambda / gamma may be NULL to use the device-resident
 * results of the last fp_adjoint_solve / fp_solve (first column). Outputs are
 * overwritten; any may be NULL. dnodes covers the vertices as ring and wake
 * nodes only: control points and normals are inputs of their own, so their
 * dependence on the nodes is the caller's chain rule. Device time:
 * fp_last_kernel_ms(FP_STAGE_VJP). */
int fp_assembly_vjp(fp_ctx* ctx, const double* lambda, const double* gamma, const double* Uinfs,
                    double* dnodes, double* dcps, double* dnormals, double* dUinfs, double* dDas,
                    double* dDbs);

/* Reverse mode of Uind! for the vortex-ring body (src/FLOWPanel_liftingbody.jl:576-661):
 * the gradient of sum_i wbar_i . Uind(targets_i) with respect to the targets
 * (dtargets 3 x m), the strengths (dstrengths N, the wake's Gamma_pi / Gamma_pj
 * included), the nodes (dnodes 3 x nnodes) and the wake directions (dDas,
 * dDbs). targets and wbar are 3 x m. Outputs are overwritten; any may be NULL. */
int fp_uind_vjp(fp_ctx* ctx, const double* strengths, const double* targets, int64_t m,
                const double* wbar, double* dtargets, double* dstrengths, double* dnodes,
                double* dDas, double* dDbs);

/* Per-launch timing of the factorisation's trailing-update kernel (the
 * tcgen05 3xTF32 kernel for FP32 factors, the SIMT FP64 kernel for FP64
 * factors), for a roofline; no counterpart in the reference. enable != 0
 * turns it on and clears the sums; every later fp_factor records CUDA events
 * on the context's stream around each such launch and adds, after the factor
 * completes, the number of launches, their device time (ms), their
 * algorithmic flops (2 m n k each) and the output elements they update (m n
 * each). */
int fp_kernel_timing(fp_ctx* ctx, int enable);
int fp_kernel_timing_read(fp_ctx* ctx, int64_t* launches, double* ms, double* flops, double* elems);

/* Timeline of the next factorisations (no counterpart in the reference): with
 * enable != 0, every fp_factor records CUDA events around each of its kernel
 * launches on all of its streams; fp_trace_read returns, for the last
 * factorisation, each launch's kernel tag (0 diagonal block, 1 block update,
 * 2 panel fix-up, 3 column strip, 4 tensor-core update, 5/6 operand splits,
 * 7 SIMT update, 8 full inverses of the diagonal block's factors),
 * its stream (0 the panel stream, 1 the trailing-update stream, 2 the third
 * stream of FP_TUNE_PANEL_GEMM 2, 3 the fourth stream of
 * FP_TUNE_REST_SPLIT) and its start
 * and end in ms from the start of the factorisation; count = launches. */
int fp_trace(fp_ctx* ctx, int enable);
int fp_trace_read(fp_ctx* ctx, int64_t cap, int* tags, int* streams, float* t0, float* t1, int64_t* count);

/* Time of the last kernel launches, for the benchmark's roofline: the device
 * time (ms) of the named stage's dominant kernel and its launch count. */
int fp_last_kernel_ms(fp_ctx* ctx, int stage, double* ms, int* launches);
#define FP_STAGE_ASSEMBLE 0
#define FP_STAGE_FACTOR 1
#define FP_STAGE_SOLVE 2
#define FP_STAGE_UIND 3
#define FP_STAGE_ADJOINT 4   /* fp_adjoint_solve */
#define FP_STAGE_VJP 5       /* fp_assembly_vjp / fp_uind_vjp */
#define FP_STAGE_POST 6      /* fp_ugradmu / fp_surface_loads */
#define FP_STAGE_PHI 7       /* fp_phi */

/* Measurement utility (no counterpart in the reference): sustained FMA
 * throughput of the FP64 (fp64 = 1) or FP32 (fp64 = 0) pipe of a device, or of
 * its FP64 tensor path (fp64 = 2: mma.sync m8n8k4 .f64), in TFLOP/s, the
 * denominator of the compute-bound kernels' roofline. */
int fp_measure_fma_peak(int device, int fp64, double* tflops);

/* Tuning knobs of a context (no counterpart in the reference; the defaults are
 * the measured best on B200):
 *   FP_TUNE_TC_STAGES   2 or 3: depth of the shared-memory ring of the tensor-core
 *                       trailing update in the static-order FP32 LU (default 2)
 *   FP_TUNE_LU_OVERLAP  1: that LU updates the columns beyond the next panel on
 *                       a second stream under the panel work (default); 0: one stream
 *   FP_TUNE_TC_TILES    output tiles per CTA of that LU's tensor-core update
 *                       (multi-tile kernel with a double-buffered accumulator);
 *                       0 (default) selects the one-tile kernel, two CTAs an SM,
 *                       which measured faster on the 12k wing (10.7 against 13.0 ms)
 *   FP_TUNE_GRAPH       1: the static-order factorisation of a problem factored
 *                       before (same sizes, buffers and knobs) replays as one CUDA
 *                       graph; 0 (default): direct launches, which measured faster
 *                       on the 12k wing (14.8 against 16.4 ms: the captured kernels
 *                       lose the panel stream's priority)
 *   FP_TUNE_TC_SMEM     bytes of shared memory each CTA of that LU's one-tile
 *                       tensor-core update reserves (0, the default: its ring
 *                       and barriers only; at most 232448): fewer update CTAs
 *                       an SM, more room for the panel kernels beside them
 *   FP_TUNE_FP64_DMMA   the FP64 LU's trailing update: 0 the SIMT FP64 kernel
 *                       (15.0 TF/s on the 12k wing); the FP64 tensor path
 *                       (mma.sync .f64) on 128 x 128 tiles, one CTA an SM:
 *                       1, 2, 3 with 8, 16 or 32 warps and 16-deep K slices
 *                       (17.0, 19.2, 19.7 TF/s), 4 with 32 warps and 32-deep
 *                       slices (20.8); on 128 x 64 tiles, two CTAs of 16 warps
 *                       an SM: 5 with 16-deep slices in 3 stages (22.4), 6
 *                       (default) with 32-deep slices in 2 stages (23.1);
 *                       all give the same results
 *   FP_TUNE_TC_SPLIT    the static-order LU's tensor-core update: 0 reads
 *                       operands split into TF32 hi / lo by the panel kernels
 *                       (32 KB a K block); 1, 2, 3: reads the unsplit FP32
 *                       operands (16 KB a K block) and splits them in shared
 *                       memory, with 3, 4 or 6 K blocks in flight a CTA
 *   FP_TUNE_TC_RED      1 (default): that update's epilogue adds to C with
 *                       red.global from the registers (factorisation 14.6 ms on
 *                       the 12k wing); 0: stages -D in shared memory for a TMA
 *                       reduce-add (15.1 ms)
 *   FP_TUNE_ASM32       1: fp_assemble for the FP32 factorisations writes the
 *                       FP32 AIC in panel-local FP32 coordinates on the
 *                       critical path (1.53 ms on the 12k wing) and the FP64
 *                       AIC (read only by the refinement) on a background
 *                       stream under the factorisation, which that pass slows
 *                       by 2.2 ms; 0 (default): one FP64 pass writes both
 *                       (2.49 ms)
 *   FP_TUNE_TC_NARROW   6 (default): the update of one column of tiles (the next
 *                       panel's columns, on the critical path) uses a 6-stage
 *                       ring; 0: the same ring as the other updates
 *   FP_TUNE_TRS2        1: the FP32 triangular sweeps of the refinement run their
 *                       chain of dependent 128-row blocks two blocks a step
 *                       (products formed once per factorisation); 0 (default):
 *                       one block a step, which measured faster on the 12k wing
 *                       (solve stage 2.38 against 2.51 ms: the two-step form
 *                       also needs the block three back, which arrives just
 *                       before the block two back). Takes effect at the next
 *                       fp_factor
 *   FP_TUNE_PANEL_GEMM  the static-order LU of the FP32 form: 2 (default) forms
 *                       the full 128 x 128 inverse of each diagonal block's L on
 *                       a third stream beside k_l21 (L21 by block substitution)
 *                       and U12 = inv(L) A12 as one triangular product; 1 forms
 *                       both full inverses on the panel stream and L21 =
 *                       A21 inv(U) as a product too; 0: block substitution
 *                       with the 32 x 32 diagonal-block inverses for both.
 *                       12k wing with the BF16-pair update: 11.7 / 12.1 /
 *                       13.1 ms of factorisation for 2 / 1 / 0 (a diagonal
 *                       block factored one pivot a step, with register tiles
 *                       and one barrier a pivot, measured 82 us a panel against
 *                       43 us and was dropped). The BF16 form always uses block
 *                       substitution
 *   FP_TUNE_TC_BF16X3   1 (default): the FP32 form's trailing update multiplies
 *                       BF16 pairs (each operand as hi + lo, C -= Ah Bl + Al Bh +
 *                       Ah Bh: three kind::f16 MMAs, half the operand bytes of
 *                       3xTF32; the 16-bit operand splits leave the refinement
 *                       at 4 steps on the 12k wing: factorisation 13.3 ->
 *                       12.1 ms); 0: 3xTF32 (TF32 pairs). Needs
 *                       FP_TUNE_PANEL_GEMM 1 or 2
 *   FP_TUNE_TC_PREFETCH 1 (default): in the tensor-core updates with the
 *                       red.global epilogue, the two warps that wait for the
 *                       accumulator prefetch the CTA's C tile into L2 during
 *                       the main loop (12k wing: update 93 -> 84 us a panel,
 *                       factorisation 11.85 -> 11.10 ms); the FP64 LU's
 *                       tensor-path update prefetches its C tile at the start
 *                       the same way; 0: the epilogues fetch C
 *   FP_TUNE_PDL         1 (default): the static-order LU's kernels (and its
 *                       BF16-pair updates) are launched with programmatic
 *                       dependent launch, so that a kernel's launch overlaps
 *                       the end of its stream's previous kernel (12k wing:
 *                       factorisation 11.12 -> 10.79 ms); 0: plain launches
 *   FP_TUNE_LU_SPLIT    1: the panel stream of the static-order LU keeps only
 *                       what the next diagonal block needs (L21 of the next
 *                       panel's rows and the update of its diagonal tile); the
 *                       third stream does L21 of the rows below and the rest of
 *                       the next panel's column beside the next k_pdiag (with
 *                       FP_TUNE_PANEL_GEMM 2; default 1: 12k wing
 *                       factorisation 10.85 -> 10.68 ms); 0: both on the panel
 *                       stream
 *   FP_TUNE_LU_FUSE     1: with the split chain, U12 of the next panel's
 *                       columns and the update of its diagonal tile (FP32, on
 *                       the FMA pipe) are one kernel; 0 (default): the tile is
 *                       updated by a tensor-core launch
 *   FP_TUNE_U12_WIDE    1: U12 of the columns beyond the next panel (BF16-pair
 *                       update) with 64 columns a CTA of 512 threads (12k
 *                       wing: 10.81 against 10.80 ms); 0 (default): 32
 *                       columns a CTA of 256 threads
 *   FP_TUNE_L21_ASYNC   1 (default): the static-order LU's L21 by a kernel that
 *                       keeps the row block and U column-major in shared memory,
 *                       staged by cp.async (12k wing: factorisation 10.81 ->
 *                       10.52 ms); 0: row-major staging through registers
 *   FP_TUNE_U12_ASYNC   1: the GEMM-form U12 kernel stages its A12 block
 *                       column-major by cp.async (K loop over 4 values a step);
 *                       0 (default): row-major through registers
 *   FP_TUNE_REST_SPLIT  split panel chain: 1: the trailing update of the
 *                       columns beyond the next panel runs as two launches,
 *                       the next panel's 128 rows first, then the rows below;
 *                       the next panel's U12 kernels wait for the first only,
 *                       and U12 of the columns beyond runs on a fourth stream
 *                       beside the second; 2: the same with the first range
 *                       on the fourth stream after that U12, so that the
 *                       second starts as soon as the U12 is done; 0
 *                       (default): one launch
 *   FP_TUNE_PDIAG_LINV  1: the diagonal-block kernel also forms the full
 *                       inverse of the block's L (no separate inverse
 *                       launch), and with the split chain L21 of the next
 *                       panel's rows runs on the third stream beside U12 of
 *                       the next panel's columns; 0 (default): a separate
 *                       launch on the third stream */
#define FP_TUNE_TC_STAGES 0
#define FP_TUNE_LU_OVERLAP 1
#define FP_TUNE_TC_TILES 2
#define FP_TUNE_GRAPH 3
#define FP_TUNE_TC_SMEM 4
#define FP_TUNE_FP64_DMMA 5
#define FP_TUNE_TC_SPLIT 6
#define FP_TUNE_TC_RED 7
#define FP_TUNE_ASM32 8
#define FP_TUNE_TC_NARROW 9
#define FP_TUNE_TRS2 10
#define FP_TUNE_PANEL_GEMM 11
#define FP_TUNE_TC_BF16X3 12
#define FP_TUNE_TC_PREFETCH 13
#define FP_TUNE_PDL 14
#define FP_TUNE_LU_SPLIT 15
#define FP_TUNE_LU_FUSE 16
#define FP_TUNE_U12_WIDE 17
#define FP_TUNE_L21_ASYNC 18
#define FP_TUNE_U12_ASYNC 19
#define FP_TUNE_REST_SPLIT 20
#define FP_TUNE_PDIAG_LINV 21
int fp_set_tuning(fp_ctx* ctx, int knob, int value);

/* Autotuner (no counterpart in the reference): times the factorisation of the
 * assembled AIC under candidate knob settings (FP_PREC_FP64: the FP64 update
 * variants of FP_TUNE_FP64_DMMA; FP_PREC_MIXED / FP_PREC_BF16: the tensor-core
 * update's epilogue, ring depth and tile kernel, or with the BF16-pair update
 * of FP_TUNE_TC_BF16X3 the ring of the next panel's update only), reps timed runs each after
 * one warm-up, and keeps the fastest for this context. The choice is cached
 * per (N, precision): a later call for the same size only applies it. The
 * context is left assembled (FP32 trials re-assemble), not factored; knobs
 * (may be NULL) receives the 10 knob values in FP_TUNE_* order. */
int fp_autotune(fp_ctx* ctx, int precision, int reps, int* knobs);

/* Measurement utility (no counterpart in the reference): number of CUDA kernels
 * this context has launched since it was created. */
int fp_kernel_launches(fp_ctx* ctx, int64_t* count);

/* Self-test utility (no counterpart in the reference): C0 - A B for seeded
 * random FP32 A (m x k), B (k x n) on device `device` by the tcgen05 3xTF32
 * kernel of the mixed-precision LU and by the SIMT FP32 kernel, each compared
 * with an FP64 evaluation; errors are max|C - C_fp64| / k (|a|, |b| <= 1). */
int fp_tc_selftest(int device, int64_t m, int64_t n, int k, double* err_tc, double* err_simt,
                   double* ms_tc);

#ifdef __cplusplus
}
#endif
#endif /* FLOWPANEL_B200_H */
