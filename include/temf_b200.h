/*
 * temf_b200.h -- C ABI of the B200-native FETD time-stepping hot path.
 *
 * Drop-in boundary for TEMF3DT's forward modelling (yxddyxzh2016/TEMF3DT,
 * Fortran 90).  The reference builds three MKL CSR matrices in mesh_process
 * and then, inside adap_euler, forms the step matrix with mkl_add_3, factors
 * and solves it with MKL cluster_sparse_solver through the module
 * pardiso_multi_real_mpi, and computes the BDF2 right-hand side with
 * mkl_sparse_d_mv.  Every one of those calls is replaced by a function below.
 *
 * Conventions (all chosen so a Fortran caller can pass its arrays unchanged
 * through ISO_C_BINDING):
 *   - every index array is 1-based, exactly as in the reference's arrays;
 *   - two-dimensional arrays are Fortran column-major with the leading
 *     dimension equal to the first extent, e.g. tet_vex(tet_num,4) is passed
 *     as a pointer to tet_num*4 ints, vertex 1 of all tets first;
 *   - all floating point data are double precision (real(8));
 *   - functions return 0 on success and a negative TEMF_E* code on failure;
 *     temf_last_error() gives the message.  No function calls exit() or
 *     stop(): the reference's `stop` on a solver error becomes a status.
 *   - one context is one GPU and one CUDA stream; a context is not
 *     thread-safe.  Device memory is owned by the context; host arrays are
 *     only read (or written) during the call.
 */
#ifndef TEMF_B200_H
#define TEMF_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define TEMF_OK 0
#define TEMF_EARG (-1)     /* invalid argument */
#define TEMF_ECUDA (-2)    /* CUDA runtime error */
#define TEMF_ESTATE (-3)   /* call out of order (e.g. solve before factor) */
#define TEMF_EINTERNAL (-4)

typedef struct temf_ctx temf_ctx;
typedef struct temf_batch temf_batch;
typedef struct temf_case temf_case;

/* ---- context --------------------------------------------------------- */
/* Create a context on CUDA device `device`. */
int temf_create(int device, temf_ctx** ctx);
int temf_destroy(temf_ctx* ctx);
/* Text of the last error of this context (never NULL). */
const char* temf_last_error(const temf_ctx* ctx);
/* Library version string. */
const char* temf_version(void);

/* ---- mesh topology helper (host only, no GPU needed) -----------------
 * Rebuilds the reference's global edge list from tet_vex:
 * model_mesh, src/FETD_FWD.f90:168-244 (unique sorted (min,max) vertex
 * pairs in lexicographic order; tet_edg by binary search; tet_drc = +1 when
 * the first local vertex of the edge has the smaller global index).
 * Call temf_mesh_count_edges first to size edg_vex. */
int temf_mesh_count_edges(int n_tets, const int* tet_vex, int* n_edges);
int temf_mesh_topology(int n_tets, const int* tet_vex, int n_edges, int* edg_vex, int* tet_edg, int* tet_drc);

/* ---- model ---------------------------------------------------------------
 * temf_set_mesh: the geometry/topology the reference keeps in type(model)
 * (src/FETD_FWD.f90:33-106): nod_cor(n_nodes,3), tet_vex(n_tets,4),
 * edg_vex(n_edges,2), tet_edg(n_tets,6), tet_drc(n_tets,6). */
int temf_set_mesh(temf_ctx* ctx, int n_nodes, const double* nod_cor, int n_tets, const int* tet_vex,
                  int n_edges, const int* edg_vex, const int* tet_edg, const int* tet_drc);
/* Per-tet conductivity (S/m) and permeability (H/m): sig_3d and mag_3d of
 * model_ctl (src/FETD_FWD.f90:347-364).  May be called again to change the
 * model; temf_assemble must then be repeated. */
int temf_set_media(temf_ctx* ctx, const double* sig_tet, const double* mu_tet);

/* Ordering + symbolic factorisation of the step-matrix pattern (once per
 * mesh; replaces the reorder/symbolic half of PARDISO phase 12,
 * src/FETD_UTILITY.f90:912-917).  Must follow temf_set_mesh. */
int temf_analyse(temf_ctx* ctx);
/* Anisotropic media ('anisotropic' section of model_ctl,
 * src/FETD_FWD.f90:368-410): per tet the row-major 3 x 3 conductivity tensor
 * sig9(9, n_tets) and permeability tensor mu9(9, n_tets) (absolute, H/m; the
 * reference builds both as dm diag(values) dm^T).  Assembly then uses
 * f_kind_ani / e_kind_ani (:853-912), the curl-curl term with the
 * elementwise reciprocal of mu9 as mesh_process passes it (:624-633).
 * Replaces temf_set_media; temf_set_media switches back to scalar media.
 * The adjoint gradient covers scalar conductivities only. */
int temf_set_media_tensor(temf_ctx* ctx, const double* sig9, const double* mu9);
/* Boundary condition (model_ctl 'boundary condition', :411-412): 0 = PEC,
 * 1 = first-order absorbing boundary, the face integrals of
 * surface_integral (:914-1007) added to the sigma-mass of every tet with a
 * boundary face (:635-640).  face_mask (n_tets bytes, bit f = local face f
 * (vertices ind_tri(f+1,:)) on the boundary) may be NULL: the faces that
 * belong to one tet are used, which is what the reference's plane test finds
 * on a convex mesh.  Takes effect at the next temf_assemble. */
int temf_set_boundary(temf_ctx* ctx, int bound_cond, const unsigned char* face_mask);

/* K1: assemble M_sigma (b_mkl) and the curl-curl matrix K (c_mkl) on the GPU:
 * mesh_process, src/FETD_FWD.f90:588-711.  Needs temf_analyse and media. */
int temf_assemble(temf_ctx* ctx);

/* Export an assembled matrix as the reference's 1-based upper-triangular CSR
 * (what mkl_to_csr returns, src/FETD_FWD.f90:1974-2004), in the original edge
 * numbering.  which: 0 = M_sigma, 1 = K.  Pass ia = ja = va = NULL to get
 * *nnz only; otherwise ia has n_edges+1 and ja/va have *nnz entries. */
int temf_get_matrix(temf_ctx* ctx, int which, int* nnz, int* ia, int* ja, double* va);

/* ---- factor / solve (the pardiso_multi_real_mpi replacement) -------------
 * temf_factor: A = 3 M_sigma + 2 dt K (mkl_add_3 call sites
 * src/FETD_FWD.f90:1288,1354) and its numeric LL^T into slot 1 or 2
 * (pardiso_direct_1, src/FETD_UTILITY.f90:879-936).  Returns 0, a negative
 * error, or a positive value = 1-based edge index of the first non-positive
 * pivot: the case in which the reference retries with mtype -2
 * (symmetric indefinite, :923-935).  The slot then holds an indefinite
 * factor A = L S L^T (S = diag(+-1), pivots that cancel below 1e-13 of their
 * diagonal entry perturbed), and temf_solve runs two steps of iterative
 * refinement with A.  temf_run stops on such a step matrix (A(dt) is SPD for
 * dt > 0); temf_solve_noalloc refuses an indefinite slot. */
int temf_factor(temf_ctx* ctx, int slot, double dt);
/* x = A^{-1} b with the factor in `slot` (pardiso_direct_2,
 * src/FETD_UTILITY.f90:938-957).  b and x are host arrays of n_edges x nrhs,
 * column-major with leading dimension ld >= n_edges (original numbering).
 * b and x may alias. */
int temf_solve(temf_ctx* ctx, int slot, int nrhs, const double* b, double* x, int ld);
/* Allocation-free solve.  It has no counterpart in the reference.  Some
 * callers cannot let a library call cudaMalloc where they solve.  Examples
 * are an application that reserves all device memory for its own pool up
 * front, a driver that must not call into the allocator while another thread
 * is capturing CUDA work, and a time loop that runs on a fixed memory budget.
 * temf_solve allocates staging and scratch buffers on first use; this call
 * allocates nothing.
 * - x_dev = A^{-1} b_dev for one right-hand side, with the factor in `slot`.
 * - b_dev and x_dev are DEVICE arrays of n_edges doubles in the original edge
 *   numbering; they may alias.  They are the caller's memory.
 * - Scratch lives in one static device array of 32 MiB that every GPU loading
 *   the library holds until the process exits.  A factor whose solve needs
 *   more returns TEMF_EARG with the byte count; use temf_solve then.
 * - The first call on a device looks the array's address up (set-up), so make
 *   that first call before another thread starts a stream capture.
 * - Every call shares the array, so calls whose GPU work overlaps (two
 *   contexts, two threads, two devices' calls are separate arrays) race.
 *   Serialise them.
 * - The call runs on the context's stream and blocks: it synchronises that
 *   stream and returns after the solve finished, with the status of its
 *   waits. */
int temf_solve_noalloc(temf_ctx* ctx, int slot, const double* b_dev, double* x_dev);
/* Forget the factor in `slot` (pardiso_direct_3, src/FETD_UTILITY.f90:959-975).
 * Device memory is kept for reuse until temf_destroy. */
int temf_release(temf_ctx* ctx, int slot);
/* y = M_sigma x for host vectors (the mkl_sparse_d_mv of the BDF2 right-hand
 * side, src/FETD_FWD.f90:1330,1367,1427).  which: 0 = M_sigma, 1 = K. */
int temf_spmv(temf_ctx* ctx, int which, int nrhs, const double* x, double* y, int ld);

/* ---- sources and receivers -----------------------------------------------
 * Sources: one edge list per right-hand-side column.  col_ptr[nrhs+1] holds
 * 0-based offsets into src_edg (1-based edge numbers) and src_drc (+1/-1):
 * src_edg/src_drc of model_ctl (src/FETD_FWD.f90:435-448).  The waveform is
 * time_const_p (src/FETD_UTILITY.f90:1050-1078): source_type 1; pulse_type
 * 1 step-on, 2 impulse, 3 step-off (DC pass first); t0 = pulse width;
 * current = amplitude.  Repeated edges in a column follow the reference's
 * assignment semantics (the last entry wins, src/FETD_FWD.f90:1507). */
int temf_set_sources(temf_ctx* ctx, int nrhs, const int* col_ptr, const int* src_edg, const int* src_drc,
                     int source_type, int pulse_type, double t0, double current);
/* Receivers: rec_tet (1-based, from p_in_tet, src/FETD_FWD.f90:1009-1049),
 * rec_cor(nrec,3), and the RHS column each receiver samples (0-based; NULL =
 * all column 0).  The interpolation and -curl operators n_arr/d_arr of
 * src/FETD_FWD.f90:712-731 are built on the GPU. */
int temf_set_receivers(temf_ctx* ctx, int nrec, const int* rec_tet, const double* rec_cor, const int* rec_rhs);
/* Copy back n_arr(rec,6,3) and d_arr(rec,6,3) in Fortran layout (checks). */
int temf_get_receiver_operators(temf_ctx* ctx, double* n_arr, double* d_arr);
/* Point location on the GPU: for each point, the first tet (in tet order)
 * whose centroid is within rec_charac and whose five 4x4 determinants share a
 * sign (p_in_tet, src/FETD_FWD.f90:1009-1049); 0 when none. */
int temf_locate_points(temf_ctx* ctx, int npts, const double* pts, double rec_charac, int* tet_out);

/* ---- the time loop ----------------------------------------------------------
 * Runs time_solver/adap_euler (src/FETD_FWD.f90:1174-1464) on the GPU:
 * sp_division, sp_double, sp_dblesize and time_maximum as in the .cntl file.
 * flags: bit 0 = reproduce the build that wrote the shipped LINUX .field
 * files (after an accepted dt-doubling trial it restarted BDF2 from
 * all_e(idx - sp_dblesize) instead of all_e(idx), src/FETD_FWD.f90:1405, and
 * advanced the time by one more old step); bit 1 = disable CUDA graphs.  forced (may be NULL): per trial 1 = accept, 0 = reject, -1 = the
 * reference's own test (used to replay a given schedule).  max_steps 0 = no
 * limit.  Results are kept in the context; see temf_result_*. */
int temf_run(temf_ctx* ctx, int sp_division, int sp_double, int sp_dblesize, double time_maximum, int flags,
             const int* forced, int n_forced, int max_steps);
/* Whole-mesh field dumps (vtkout, src/FETD_FWD.f90:1642-1864): the following
 * temf_run evaluates E and D at every tet's centroid at every output row,
 * accumulates B = sum D dt, and keeps E, D, B of the first row at or after
 * each of the n_times times (at most 30; 0 turns the dumps off).  One RHS
 * column; not in batches.  temf_result_mesh_fields: snapshot `index` of the
 * last run as fields(tets, 9) row-major = Ex Ey Ez Dx Dy Dz Bx By Bz, and
 * whether the run reached it (*done). */
int temf_set_mesh_fields(temf_ctx* ctx, int n_times, const double* times);
int temf_result_mesh_fields(temf_ctx* ctx, int index, double* fields, int* done);
/* Number of output rows of the last run (the rows of the .field file). */
int temf_result_rows(temf_ctx* ctx, int* rows);
/* Output rows: step(rows), time(rows), dt(rows) and fields(9, nrec, rows)
 * = ex ey ez dBx/dt dBy/dt dBz/dt bx by bz per receiver, as a_f of
 * solution_output (src/FETD_FWD.f90:1530-1622), Fortran order (component
 * fastest).  Any pointer may be NULL. */
int temf_result_get(temf_ctx* ctx, int* step, double* time, double* dt, double* fields);
/* Trial statistics: number of trials, errors and accept flags (NULL ok). */
int temf_result_trials(temf_ctx* ctx, int* n_trials, double* errors, int* accepted);
/* Time-gate interpolation (.field2, src/FETD_FWD.f90:1625-1640): for each of
 * n_gates times, fields(9, nrec, n_gates) and a done flag. */
int temf_result_gates(temf_ctx* ctx, int n_gates, const double* gates, double* fields, int* done);
/* Timing of the last run in milliseconds (CUDA events): factorisations,
 * stepping (SpMV+solve+receivers), whole run; counts of factorisations,
 * solves and kernel launches. */
int temf_result_timing(temf_ctx* ctx, double* ms_factor, double* ms_steps, double* ms_total, int* n_factor,
                       int* n_solve, long long* n_launch);

/* ---- sweep schedule autotuner ------------------------------------------------
 * No reference counterpart.  The persistent triangular-solve sweeps hand the
 * supernodes below a split level (counted from the leaves) to CTAs through a
 * ready queue, and claim the ones above it in schedule order with their panel
 * copies issued before the dependency waits.  temf_tune_solve times one solve
 * of nrhs columns (right-hand side all ones; nrhs > 1 tunes the 64-column
 * block sweeps) with the factor in slot 1 or 2 for up to 8 candidate levels
 * and keeps the fastest; temf_run tunes once on its first factorisation if
 * nothing was tuned since temf_analyse.  cand_split/cand_ms (may be NULL)
 * receive the candidates.  temf_solve_schedule reports the level in use. */
int temf_tune_solve(temf_ctx* ctx, int slot, int nrhs, int* split, int* n_cand, int* cand_split, double* cand_ms);
int temf_solve_schedule(temf_ctx* ctx, int nrhs, int* split, int* tuned);
/* The single-column sweeps (temf_solve, temf_run) first sweep the bottom of
 * the supernodal tree as whole subtrees, one warp each: the supernodes below
 * a subtree level, with no waits; the persistent task sweeps cover the rest.
 * Above the queue split, the column blocks of a wide supernode (one per
 * level) are swept by one leader task that forwards the rows inside the run
 * through shared memory instead of handing each block to another CTA
 * (run_leaders = 1).  For nrhs = 1, temf_tune_solve also picks the subtree
 * level (0 = none, or levels that leave at least one subtree per SM) before
 * the queue split, then whether to use run leaders, and reports the split
 * candidates at the chosen level.  temf_set_solve_plan sets the plan
 * explicitly (checked on the host, marked tuned); temf_solve_plan reports the
 * plan in use and its number of subtrees.  No reference counterpart. */
int temf_set_solve_plan(temf_ctx* ctx, int tree_level, int split, int run_leaders);
int temf_solve_plan(temf_ctx* ctx, int* tree_level, int* split, int* run_leaders, int* n_trees, int* tuned);
/* Failure detection of the device waits.  No reference counterpart.  Every
 * wait of the persistent sweeps on a flag another CTA sets is bounded: after
 * `spins` polls (0: the default, about a second) it gives up, records which
 * wait it was in an error word and lets the kernel finish, so the context
 * stays usable; temf_solve / temf_run then return TEMF_ESTATE ("a
 * triangular-solve wait timed out (code k)").  inject_unmet_wait = 1 makes
 * the next single-column solve outside stream capture expect one input more
 * than any task provides for the last supernode, so that one wait cannot be
 * met (a test of this path; it is consumed by that solve). */
int temf_set_wait_limit(temf_ctx* ctx, int spins, int inject_unmet_wait);

/* ---- profiling aid -------------------------------------------------------------
 * No reference counterpart.  One single-column solve (right-hand side all
 * ones) with the factor in slot 1 or 2, recording per task of the persistent
 * sweeps: start, dependency satisfied, end (GPU global timer, ns), SM id,
 * supernode, kind (0 diagonal, 1 row chunk, 2 a whole subtree swept by one
 * warp: supernode = its root, first row = its first supernode), first row,
 * supernode level -- 8 words per task, the n_fwd forward tasks first (forward
 * subtrees, then tasks), then the n_bwd backward ones (tasks, then
 * subtrees).  With out = NULL only the counts are returned. */
int temf_solve_timeline(temf_ctx* ctx, int slot, long long cap, unsigned long long* out, int* n_fwd, int* n_bwd);

/* ---- adjoint gradient --------------------------------------------------------
 * No reference counterpart: the reference's inversion module (inv_modeling)
 * ships only as compiled objects.  These entries give the gradient of a
 * misfit of the receiver output with respect to the conductivities.
 *
 * temf_adjoint_record: the following temf_run calls record their solve graph
 * and keep, every checkpoint_every solves and wherever dt changes, a
 * checkpoint of the BDF2 history (2*sp_dblesize+2 state vectors of n doubles
 * each).  A recording run launches its kernels one by one (no CUDA graphs),
 * needs one RHS column and pulse type 1 or 2.  0 turns recording off and
 * frees the checkpoints.
 *
 * temf_adjoint: reverse sweep over the recorded run.  dJ_dfields(9, nrec,
 * rows) is dJ/d(fields) in the layout temf_result_get returns (the b columns
 * are chained back onto dB/dt).  tet_cell(n_tets): 1-based inversion cell of
 * each tet, 0 = not in the grid.  Writes grad_logsigma(ncell) = dJ/dlog sigma_c
 * = sum over the cell's tets of sigma_t dJ/dsigma_t, and, if grad_sigma is
 * not NULL, grad_sigma(n_tets) = dJ/dsigma_t.  Uses factor slot 1 (the
 * factor held there is released).  tet_cell and grad_logsigma may be NULL
 * together.  Changing the media (temf_set_media) discards the recording. */
int temf_adjoint_record(temf_ctx* ctx, int checkpoint_every);
int temf_adjoint(temf_ctx* ctx, const double* dJ_dfields, int ncell, const int* tet_cell, double* grad_logsigma,
                 double* grad_sigma);
/* Timing of the last adjoint sweep: ms[0] whole sweep, ms[1] factorisations;
 * counts[0] solve-graph nodes, counts[1] checkpoint blocks, counts[2]
 * factorisations, counts[3] kernel launches.  Either pointer may be NULL. */
int temf_adjoint_timing(temf_ctx* ctx, double* ms, long long* counts);

/* ---- many models at once ------------------------------------------------------
 * No reference counterpart (the reference runs one model per process).  A
 * batch steps several independent models -- each a context prepared up to
 * temf_set_sources/temf_set_receivers, one RHS column, pulse type 1 or 2 --
 * through the adaptive time loop in lockstep on one GPU: every model keeps
 * its own dt schedule, factors and accept/reject decisions, while the
 * triangular solves of all models in a step run as one merged persistent
 * forward and one backward kernel.  Results land in each model's context
 * (temf_result_*).  The contexts must share a device and outlive the batch.
 *
 * temf_batch_run flags: bit 0 = legacy LINUX schedule (as temf_run), bit 1 =
 * no CUDA graphs, bit 2 = autotune: before the first step the candidate
 * merge orders (0 proportional interleave, 1 level-aligned, 2 one model after
 * another) and resident-CTA fractions (100 %, 67 %) are timed on one merged
 * solve and the fastest is kept for this and later runs.  max_steps 0 = no
 * limit.  temf_batch_timing: ms[0..3] = whole run, factorisations, stepping,
 * tuning; counts[0..2] = lockstep steps, kernel launches, merged solves.
 * temf_batch_tuning returns 1 if tuned (order, grid_pct and, if not NULL,
 * the six candidate times in ms), 0 if not. */
int temf_batch_create(temf_ctx* const* models, int n_models, temf_batch** batch);
int temf_batch_destroy(temf_batch* batch);
const char* temf_batch_last_error(const temf_batch* batch);
int temf_batch_run(temf_batch* batch, int sp_division, int sp_double, int sp_dblesize, double time_maximum,
                   int flags, int max_steps);
int temf_batch_timing(temf_batch* batch, double* ms, long long* counts);
int temf_batch_tuning(temf_batch* batch, int* order, int* grid_pct, double* candidate_ms);
int temf_batch_set_tuning(temf_batch* batch, int order, int grid_pct);

/* Options of the next temf_analyse (no reference counterpart; MKL's ordering
 * has its own knobs in iparm): nested-dissection leaf size (default 96) and
 * supernode amalgamation (0 none, 1: merge while few explicit zeros are
 * added, 2 (default): also merge small supernodes harder, for fewer and
 * larger solve tasks, 3: merge up to 64 columns at 25 % explicit zeros; on
 * the 1.2M-edge mesh 18 % fewer supernodes for 0.8 % more nnz(L)). */
int temf_set_analysis_options(temf_ctx* ctx, int leaf_size, int amalg_level);

/* ---- statistics of the symbolic analysis ----------------------------------
 * stats[0..9] = n, nnz(A full), supernodes, levels, nnz(L), stored doubles,
 * factor flops, update tiles, seconds ordering, seconds symbolic. */
int temf_analysis_stats(temf_ctx* ctx, double* stats);

/* Host-only ordering + symbolic analysis of a symmetric pattern (no GPU
 * needed): 0-based adjacency without the diagonal (xadj[n+1], adj), one point
 * per unknown in xyz(3,n) (x,y,z of each unknown contiguous).  perm_out[new]
 * = old (0-based).  stats[0..8] = n, supernodes, levels, nnz(L) held by the
 * supernodes, stored doubles, factor flops, seconds ordering, seconds
 * symbolic, structural nnz(L) (sum of column counts). */
int temf_symbolic_host(int n, const long long* xadj, const int* adj, const double* xyz, int* perm_out,
                       double* stats);

/* Host-only check of an analysis (no GPU needed): the supernode row lists (ascending, below the diagonal block, every child row
 * inside its parent's panel), then the triangular-solve schedules replayed,
 * claimed in order and through the ready queue, for both chunk heights.
 * Returns 0, or 1 with the first violation in msg. */
int temf_schedule_check(int n, const long long* xadj, const int* adj, const double* xyz, char* msg, int msg_len);

/* ---- PARDISO-compatible shim ------------------------------------------------
 * Same argument meaning as the reference's module pardiso_multi_real_mpi
 * (src/FETD_UTILITY.f90:826-1028) so adap_euler can keep its five calls.
 * direct_1 takes the 1-based upper CSR (ia, ja, va) of A; its pattern must be
 * the assembled step-matrix pattern of the mesh set on the context (the
 * pattern mkl_add_3 produces), which is checked.  A matrix that is not
 * positive definite is factored in the indefinite mode as with temf_factor;
 * direct_1 then returns the first non-positive pivot column (> 0), where the
 * reference prints its "CHANGE TO INDEFINITE MODE" warning, and direct_2
 * refines its solves. */
/* pardiso_checker (src/FETD_UTILITY.f90:993-1027), host only: the CSR
 * structure checks the reference asks of MKL's sparse matrix checker (ia(1) =
 * 1, ia(n+1)-1 = nnz, ia non-decreasing, ja in 1..n and strictly ascending per
 * row, upper triangle when symm != 0).  *checker = 1 if the structure is
 * valid, else 0 with the first violation in msg; returns 0, or TEMF_EARG for
 * null pointers.  temf_pardiso_direct_1 runs the same checks and fails with
 * TEMF_EARG where the reference stops with "matrix error!". */
int temf_pardiso_checker(int symm, int n, int nnz, const int* ia, const int* ja, int* checker, char* msg,
                         int msg_len);
int temf_pardiso_alloc(temf_ctx* ctx, int max_matrix);
int temf_pardiso_direct_1(temf_ctx* ctx, int num_m, int symm, int n, int nnz, const int* ia, const int* ja,
                          const double* va);
int temf_pardiso_direct_2(temf_ctx* ctx, int num_m, const double* b, double* x);
int temf_pardiso_direct_3(temf_ctx* ctx, int num_m);
int temf_pardiso_dealloc(temf_ctx* ctx);

/* ---- the reference's file front end (./FETD -f ROOT) --------------------------
 * Host only, except temf_case_load / temf_case_run, which drive a context.
 *
 * temf_case_read: ROOT.mesh (model_mesh, MEDIT sections Vertices / Edges
 * (tagged edges = source segments) / Tetrahedra, src/FETD_FWD.f90:112-166) and
 * ROOT.cntl (model_ctl keywords, :284-497, with its completeness test,
 * :490-497).  On failure returns TEMF_EARG with the reason in msg. */
int temf_case_read(const char* root, temf_case** out, char* msg, int msg_len);
int temf_case_free(temf_case* cs);
/* sizes[0..6] = nodes, tets, source segments, receivers, isotropic domains,
 * anisotropic domains, time points (-1 when the cntl has none). */
int temf_case_sizes(const temf_case* cs, int* sizes);
/* The mesh in the reference's Fortran layouts: nod_cor(nodes,3),
 * tet_vex(tets,4), tet_phy(tets), src_vex(segments,2), src_phy(segments);
 * 1-based vertex numbers.  NULL arrays are skipped. */
int temf_case_mesh(const temf_case* cs, double* nod_cor, int* tet_vex, int* tet_phy, int* src_vex, int* src_phy);
/* The control: ints[10] = bound_cond, src_num, source_type, pulse_type,
 * sp_mthd, sp_division, sp_double, sp_dblesize, vtkout, output mask (bit k =
 * column k of ex ey ez dx dy dz bx by bz); reals[4] = rec_charac, t0,
 * current, time_maximum; rec_cor(receivers,3); time_points. */
int temf_case_control(const temf_case* cs, int* ints, double* reals, double* rec_cor, double* time_points);
/* Media per tet (src/FETD_FWD.f90:347-409): *aniso = 0: sig(tets) and
 * mu(tets) = mu_r mu0; *aniso = 1: row-major 3 x 3 tensors (tets,9), the
 * rotation as the reference builds it.  TEMF_EARG if a tet's physical domain
 * is not in the cntl. */
int temf_case_media(const temf_case* cs, double* sig, double* mu, int* aniso);
/* .field rows as solution_output writes them (src/FETD_FWD.f90:1623,
 * format i6, e15.5, 2x, nrec(n e15.5, 2x), n = selected columns): steps(rows),
 * times(rows), fields(9, nrec, rows) as temf_result_get returns them,
 * output_mask[9] (non-zero = written).  Fortran E15.5 numbers. */
int temf_case_write_rows(const char* path, int rows, int nrec, const int* steps, const double* times,
                         const double* fields, const int* output_mask);
/* Whole-mesh field dumps (vtkout, src/FETD_FWD.f90:1642-1864), host parts.
 * temf_case_vtk_times: the vtkout times of the cntl (*n of them; times may
 * be NULL).  temf_mesh_fields_host: vtk_field_save's E and D of an edge
 * vector e(n_edges) at every tet's centroid, fields(tets, 6) row-major =
 * Ex Ey Ez Dx Dy Dz (mesh arrays in the Fortran layouts of temf_set_mesh).
 * temf_case_write_msh: msh_output -- a copy of the Gmsh 4.1 file src_msh
 * with one $ElementData block (absolute values, i10 e16.8) per output column
 * selected in the cntl, from fields(tets, 9) row-major = E, D, B; the tets
 * are matched to the file's tetrahedron elements in order. */
int temf_case_vtk_times(const temf_case* cs, int* n, double* times);
int temf_mesh_fields_host(int n_nodes, const double* nod_cor, int n_tets, const int* tet_vex, const int* tet_edg,
                          const int* tet_drc, int n_edges, const double* e, double* fields);
int temf_case_write_msh(const temf_case* cs, const char* src_msh, const char* dst_msh, const double* fields, char* msg,
                        int msg_len);
/* mesh_process and the source/receiver set-up on a fresh context: edge
 * topology, mesh, media, boundary, analysis, assembly, src_edg/src_drc (+1,
 * last -1, src/FETD_FWD.f90:435-448), receiver location and operators. */
int temf_case_load(temf_case* cs, temf_ctx* ctx, char* msg, int msg_len);
/* ROOT.field from the last temf_run of ctx, and ROOT.field2 (the time_points
 * rows the run reached, numbered from 1) when the cntl has time_points. */
int temf_case_write(const temf_case* cs, temf_ctx* ctx, const char* root, char* msg, int msg_len);
/* `./FETD -f ROOT` on GPU `device`: read, load, temf_run (flags as there),
 * write ROOT.field(2); with vtkout times in the cntl and ROOT.msh present,
 * also ROOT_i.msh for each time the run reached (msh_output). */
int temf_case_run(const char* root, int device, int flags, char* msg, int msg_len);

#ifdef __cplusplus
}
#endif
#endif /* TEMF_B200_H */
