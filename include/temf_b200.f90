! ISO_C_BINDING interface to libtemf_b200.so: one bind(C) interface per
! entry point of temf_b200.h, with the same argument order and meaning.
! Context and batch handles are type(c_ptr) passed by value; arrays are
! assumed-size, so the reference's allocatable arrays (1-based indices,
! column-major real(8)) pass unchanged.  Strings come back as C pointers
! (c_f_pointer turns them into Fortran strings).  temf_solve_noalloc takes
! device addresses.  The status codes mirror TEMF_OK / TEMF_E* of the header.
module temf_b200
  use iso_c_binding
  implicit none
  integer(c_int), parameter :: TEMF_OK = 0, TEMF_EARG = -1, TEMF_ECUDA = -2, TEMF_ESTATE = -3, &
                               TEMF_EINTERNAL = -4
  interface
    integer(c_int) function temf_create(device, ctx) bind(C, name="temf_create")
      import; integer(c_int), value :: device; type(c_ptr) :: ctx
    end function
    integer(c_int) function temf_destroy(ctx) bind(C, name="temf_destroy")
      import; type(c_ptr), value :: ctx
    end function
    type(c_ptr) function temf_last_error(ctx) bind(C, name="temf_last_error")
      import; type(c_ptr), value :: ctx
    end function
    type(c_ptr) function temf_version() bind(C, name="temf_version")
      import
    end function
    integer(c_int) function temf_mesh_count_edges(n_tets, tet_vex, n_edges) &
        bind(C, name="temf_mesh_count_edges")
      import; integer(c_int), value :: n_tets; integer(c_int) :: tet_vex(*); integer(c_int) :: n_edges
    end function
    integer(c_int) function temf_mesh_topology(n_tets, tet_vex, n_edges, edg_vex, tet_edg, tet_drc) &
        bind(C, name="temf_mesh_topology")
      import; integer(c_int), value :: n_tets; integer(c_int) :: tet_vex(*); integer(c_int), value :: n_edges 
      integer(c_int) :: edg_vex(*); integer(c_int) :: tet_edg(*); integer(c_int) :: tet_drc(*)
    end function
    integer(c_int) function temf_set_mesh(ctx, n_nodes, nod_cor, n_tets, tet_vex, n_edges, edg_vex, tet_edg, tet_drc) &
        bind(C, name="temf_set_mesh")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: n_nodes; real(c_double) :: nod_cor(*) 
      integer(c_int), value :: n_tets; integer(c_int) :: tet_vex(*); integer(c_int), value :: n_edges 
      integer(c_int) :: edg_vex(*); integer(c_int) :: tet_edg(*); integer(c_int) :: tet_drc(*)
    end function
    integer(c_int) function temf_set_media(ctx, sig_tet, mu_tet) bind(C, name="temf_set_media")
      import; type(c_ptr), value :: ctx; real(c_double) :: sig_tet(*); real(c_double) :: mu_tet(*)
    end function
    integer(c_int) function temf_analyse(ctx) bind(C, name="temf_analyse")
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function temf_set_media_tensor(ctx, sig9, mu9) bind(C, name="temf_set_media_tensor")
      import; type(c_ptr), value :: ctx; real(c_double) :: sig9(*); real(c_double) :: mu9(*)
    end function
    integer(c_int) function temf_set_boundary(ctx, bound_cond, face_mask) bind(C, name="temf_set_boundary")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: bound_cond; type(c_ptr), value :: face_mask
    end function
    integer(c_int) function temf_assemble(ctx) bind(C, name="temf_assemble")
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function temf_get_matrix(ctx, which, nnz, ia, ja, va) bind(C, name="temf_get_matrix")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: which; integer(c_int) :: nnz 
      integer(c_int) :: ia(*); integer(c_int) :: ja(*); real(c_double) :: va(*)
    end function
    integer(c_int) function temf_factor(ctx, slot, dt) bind(C, name="temf_factor")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: slot; real(c_double), value :: dt
    end function
    integer(c_int) function temf_solve(ctx, slot, nrhs, b, x, ld) bind(C, name="temf_solve")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: slot; integer(c_int), value :: nrhs 
      real(c_double) :: b(*); real(c_double) :: x(*); integer(c_int), value :: ld
    end function
    integer(c_int) function temf_solve_noalloc(ctx, slot, b_dev, x_dev) bind(C, name="temf_solve_noalloc")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: slot; type(c_ptr), value :: b_dev 
      type(c_ptr), value :: x_dev
    end function
    integer(c_int) function temf_release(ctx, slot) bind(C, name="temf_release")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: slot
    end function
    integer(c_int) function temf_spmv(ctx, which, nrhs, x, y, ld) bind(C, name="temf_spmv")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: which; integer(c_int), value :: nrhs 
      real(c_double) :: x(*); real(c_double) :: y(*); integer(c_int), value :: ld
    end function
    integer(c_int) function temf_set_sources(ctx, nrhs, col_ptr, src_edg, src_drc, source_type, pulse_type, t0, current) &
        bind(C, name="temf_set_sources")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: nrhs; integer(c_int) :: col_ptr(*) 
      integer(c_int) :: src_edg(*); integer(c_int) :: src_drc(*); integer(c_int), value :: source_type 
      integer(c_int), value :: pulse_type; real(c_double), value :: t0; real(c_double), value :: current
    end function
    integer(c_int) function temf_set_receivers(ctx, nrec, rec_tet, rec_cor, rec_rhs) &
        bind(C, name="temf_set_receivers")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: nrec; integer(c_int) :: rec_tet(*) 
      real(c_double) :: rec_cor(*); integer(c_int) :: rec_rhs(*)
    end function
    integer(c_int) function temf_get_receiver_operators(ctx, n_arr, d_arr) &
        bind(C, name="temf_get_receiver_operators")
      import; type(c_ptr), value :: ctx; real(c_double) :: n_arr(*); real(c_double) :: d_arr(*)
    end function
    integer(c_int) function temf_locate_points(ctx, npts, pts, rec_charac, tet_out) &
        bind(C, name="temf_locate_points")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: npts; real(c_double) :: pts(*) 
      real(c_double), value :: rec_charac; integer(c_int) :: tet_out(*)
    end function
    integer(c_int) function temf_run(ctx, sp_division, sp_double, sp_dblesize, time_maximum, flags, forced, n_forced, max_steps) &
        bind(C, name="temf_run")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: sp_division; integer(c_int), value :: sp_double 
      integer(c_int), value :: sp_dblesize; real(c_double), value :: time_maximum; integer(c_int), value :: flags 
      integer(c_int) :: forced(*); integer(c_int), value :: n_forced; integer(c_int), value :: max_steps
    end function
    integer(c_int) function temf_set_mesh_fields(ctx, n_times, times) bind(C, name="temf_set_mesh_fields")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: n_times; real(c_double) :: times(*)
    end function
    integer(c_int) function temf_result_mesh_fields(ctx, index, fields, done) &
        bind(C, name="temf_result_mesh_fields")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: index; real(c_double) :: fields(*) 
      integer(c_int) :: done
    end function
    integer(c_int) function temf_result_rows(ctx, rows) bind(C, name="temf_result_rows")
      import; type(c_ptr), value :: ctx; integer(c_int) :: rows
    end function
    integer(c_int) function temf_result_get(ctx, step, time, dt, fields) bind(C, name="temf_result_get")
      import; type(c_ptr), value :: ctx; integer(c_int) :: step(*); real(c_double) :: time(*) 
      real(c_double) :: dt(*); real(c_double) :: fields(*)
    end function
    integer(c_int) function temf_result_trials(ctx, n_trials, errors, accepted) &
        bind(C, name="temf_result_trials")
      import; type(c_ptr), value :: ctx; integer(c_int) :: n_trials; real(c_double) :: errors(*) 
      integer(c_int) :: accepted(*)
    end function
    integer(c_int) function temf_result_gates(ctx, n_gates, gates, fields, done) &
        bind(C, name="temf_result_gates")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: n_gates; real(c_double) :: gates(*) 
      real(c_double) :: fields(*); integer(c_int) :: done(*)
    end function
    integer(c_int) function temf_result_timing(ctx, ms_factor, ms_steps, ms_total, n_factor, n_solve, n_launch) &
        bind(C, name="temf_result_timing")
      import; type(c_ptr), value :: ctx; real(c_double) :: ms_factor; real(c_double) :: ms_steps 
      real(c_double) :: ms_total; integer(c_int) :: n_factor; integer(c_int) :: n_solve 
      integer(c_long_long) :: n_launch
    end function
    integer(c_int) function temf_tune_solve(ctx, slot, nrhs, split, n_cand, cand_split, cand_ms) &
        bind(C, name="temf_tune_solve")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: slot; integer(c_int), value :: nrhs 
      integer(c_int) :: split; integer(c_int) :: n_cand; integer(c_int) :: cand_split(*); real(c_double) :: cand_ms(*)
    end function
    integer(c_int) function temf_solve_schedule(ctx, nrhs, split, tuned) bind(C, name="temf_solve_schedule")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: nrhs; integer(c_int) :: split; integer(c_int) :: tuned
    end function
    integer(c_int) function temf_set_solve_plan(ctx, tree_level, split, run_leaders) &
        bind(C, name="temf_set_solve_plan")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: tree_level; integer(c_int), value :: split
      integer(c_int), value :: run_leaders
    end function
    integer(c_int) function temf_solve_plan(ctx, tree_level, split, run_leaders, n_trees, tuned) &
        bind(C, name="temf_solve_plan")
      import; type(c_ptr), value :: ctx; integer(c_int) :: tree_level; integer(c_int) :: split
      integer(c_int) :: run_leaders; integer(c_int) :: n_trees; integer(c_int) :: tuned
    end function
    integer(c_int) function temf_set_wait_limit(ctx, spins, inject_unmet_wait) bind(C, name="temf_set_wait_limit")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: spins; integer(c_int), value :: inject_unmet_wait
    end function
    integer(c_int) function temf_solve_timeline(ctx, slot, cap, out, n_fwd, n_bwd) &
        bind(C, name="temf_solve_timeline")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: slot; integer(c_long_long), value :: cap 
      integer(c_long_long) :: out(*); integer(c_int) :: n_fwd; integer(c_int) :: n_bwd
    end function
    integer(c_int) function temf_adjoint_record(ctx, checkpoint_every) bind(C, name="temf_adjoint_record")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: checkpoint_every
    end function
    integer(c_int) function temf_adjoint(ctx, dJ_dfields, ncell, tet_cell, grad_logsigma, grad_sigma) &
        bind(C, name="temf_adjoint")
      import; type(c_ptr), value :: ctx; real(c_double) :: dJ_dfields(*); integer(c_int), value :: ncell 
      integer(c_int) :: tet_cell(*); real(c_double) :: grad_logsigma(*); real(c_double) :: grad_sigma(*)
    end function
    integer(c_int) function temf_adjoint_timing(ctx, ms, counts) bind(C, name="temf_adjoint_timing")
      import; type(c_ptr), value :: ctx; real(c_double) :: ms(*); integer(c_long_long) :: counts(*)
    end function
    integer(c_int) function temf_batch_create(models, n_models, batch) bind(C, name="temf_batch_create")
      import; type(c_ptr) :: models(*); integer(c_int), value :: n_models; type(c_ptr) :: batch
    end function
    integer(c_int) function temf_batch_destroy(batch) bind(C, name="temf_batch_destroy")
      import; type(c_ptr), value :: batch
    end function
    type(c_ptr) function temf_batch_last_error(batch) bind(C, name="temf_batch_last_error")
      import; type(c_ptr), value :: batch
    end function
    integer(c_int) function temf_batch_run(batch, sp_division, sp_double, sp_dblesize, time_maximum, flags, max_steps) &
        bind(C, name="temf_batch_run")
      import; type(c_ptr), value :: batch; integer(c_int), value :: sp_division; integer(c_int), value :: sp_double 
      integer(c_int), value :: sp_dblesize; real(c_double), value :: time_maximum; integer(c_int), value :: flags 
      integer(c_int), value :: max_steps
    end function
    integer(c_int) function temf_batch_timing(batch, ms, counts) bind(C, name="temf_batch_timing")
      import; type(c_ptr), value :: batch; real(c_double) :: ms(*); integer(c_long_long) :: counts(*)
    end function
    integer(c_int) function temf_batch_tuning(batch, order, grid_pct, candidate_ms) &
        bind(C, name="temf_batch_tuning")
      import; type(c_ptr), value :: batch; integer(c_int) :: order; integer(c_int) :: grid_pct 
      real(c_double) :: candidate_ms(*)
    end function
    integer(c_int) function temf_batch_set_tuning(batch, order, grid_pct) &
        bind(C, name="temf_batch_set_tuning")
      import; type(c_ptr), value :: batch; integer(c_int), value :: order; integer(c_int), value :: grid_pct
    end function
    integer(c_int) function temf_set_analysis_options(ctx, leaf_size, amalg_level) &
        bind(C, name="temf_set_analysis_options")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: leaf_size; integer(c_int), value :: amalg_level
    end function
    integer(c_int) function temf_analysis_stats(ctx, stats) bind(C, name="temf_analysis_stats")
      import; type(c_ptr), value :: ctx; real(c_double) :: stats(*)
    end function
    integer(c_int) function temf_symbolic_host(n, xadj, adj, xyz, perm_out, stats) &
        bind(C, name="temf_symbolic_host")
      import; integer(c_int), value :: n; integer(c_long_long) :: xadj(*); integer(c_int) :: adj(*) 
      real(c_double) :: xyz(*); integer(c_int) :: perm_out(*); real(c_double) :: stats(*)
    end function
    integer(c_int) function temf_schedule_check(n, xadj, adj, xyz, msg, msg_len) &
        bind(C, name="temf_schedule_check")
      import; integer(c_int), value :: n; integer(c_long_long) :: xadj(*); integer(c_int) :: adj(*) 
      real(c_double) :: xyz(*); character(kind=c_char) :: msg(*); integer(c_int), value :: msg_len
    end function
    integer(c_int) function temf_pardiso_checker(symm, n, nnz, ia, ja, checker, msg, msg_len) &
        bind(C, name="temf_pardiso_checker")
      import; integer(c_int), value :: symm; integer(c_int), value :: n; integer(c_int), value :: nnz 
      integer(c_int) :: ia(*); integer(c_int) :: ja(*); integer(c_int) :: checker; character(kind=c_char) :: msg(*) 
      integer(c_int), value :: msg_len
    end function
    integer(c_int) function temf_pardiso_alloc(ctx, max_matrix) bind(C, name="temf_pardiso_alloc")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: max_matrix
    end function
    integer(c_int) function temf_pardiso_direct_1(ctx, num_m, symm, n, nnz, ia, ja, va) &
        bind(C, name="temf_pardiso_direct_1")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: num_m; integer(c_int), value :: symm 
      integer(c_int), value :: n; integer(c_int), value :: nnz; integer(c_int) :: ia(*); integer(c_int) :: ja(*) 
      real(c_double) :: va(*)
    end function
    integer(c_int) function temf_pardiso_direct_2(ctx, num_m, b, x) bind(C, name="temf_pardiso_direct_2")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: num_m; real(c_double) :: b(*); real(c_double) :: x(*)
    end function
    integer(c_int) function temf_pardiso_direct_3(ctx, num_m) bind(C, name="temf_pardiso_direct_3")
      import; type(c_ptr), value :: ctx; integer(c_int), value :: num_m
    end function
    integer(c_int) function temf_pardiso_dealloc(ctx) bind(C, name="temf_pardiso_dealloc")
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function temf_case_read(root, out, msg, msg_len) bind(C, name="temf_case_read")
      import; character(kind=c_char) :: root(*); type(c_ptr) :: out; character(kind=c_char) :: msg(*) 
      integer(c_int), value :: msg_len
    end function
    integer(c_int) function temf_case_free(cs) bind(C, name="temf_case_free")
      import; type(c_ptr), value :: cs
    end function
    integer(c_int) function temf_case_sizes(cs, sizes) bind(C, name="temf_case_sizes")
      import; type(c_ptr), value :: cs; integer(c_int) :: sizes(*)
    end function
    integer(c_int) function temf_case_mesh(cs, nod_cor, tet_vex, tet_phy, src_vex, src_phy) &
        bind(C, name="temf_case_mesh")
      import; type(c_ptr), value :: cs; real(c_double) :: nod_cor(*); integer(c_int) :: tet_vex(*) 
      integer(c_int) :: tet_phy(*); integer(c_int) :: src_vex(*); integer(c_int) :: src_phy(*)
    end function
    integer(c_int) function temf_case_control(cs, ints, reals, rec_cor, time_points) &
        bind(C, name="temf_case_control")
      import; type(c_ptr), value :: cs; integer(c_int) :: ints(*); real(c_double) :: reals(*) 
      real(c_double) :: rec_cor(*); real(c_double) :: time_points(*)
    end function
    integer(c_int) function temf_case_media(cs, sig, mu, aniso) bind(C, name="temf_case_media")
      import; type(c_ptr), value :: cs; real(c_double) :: sig(*); real(c_double) :: mu(*); integer(c_int) :: aniso
    end function
    integer(c_int) function temf_case_write_rows(path, rows, nrec, steps, times, fields, output_mask) &
        bind(C, name="temf_case_write_rows")
      import; character(kind=c_char) :: path(*); integer(c_int), value :: rows; integer(c_int), value :: nrec 
      integer(c_int) :: steps(*); real(c_double) :: times(*); real(c_double) :: fields(*) 
      integer(c_int) :: output_mask(*)
    end function
    integer(c_int) function temf_case_vtk_times(cs, n, times) bind(C, name="temf_case_vtk_times")
      import; type(c_ptr), value :: cs; integer(c_int) :: n; real(c_double) :: times(*)
    end function
    integer(c_int) function temf_mesh_fields_host(n_nodes, nod_cor, n_tets, tet_vex, tet_edg, tet_drc, n_edges, e, fields) &
        bind(C, name="temf_mesh_fields_host")
      import; integer(c_int), value :: n_nodes; real(c_double) :: nod_cor(*); integer(c_int), value :: n_tets 
      integer(c_int) :: tet_vex(*); integer(c_int) :: tet_edg(*); integer(c_int) :: tet_drc(*) 
      integer(c_int), value :: n_edges; real(c_double) :: e(*); real(c_double) :: fields(*)
    end function
    integer(c_int) function temf_case_write_msh(cs, src_msh, dst_msh, fields, msg, msg_len) &
        bind(C, name="temf_case_write_msh")
      import; type(c_ptr), value :: cs; character(kind=c_char) :: src_msh(*); character(kind=c_char) :: dst_msh(*) 
      real(c_double) :: fields(*); character(kind=c_char) :: msg(*); integer(c_int), value :: msg_len
    end function
    integer(c_int) function temf_case_load(cs, ctx, msg, msg_len) bind(C, name="temf_case_load")
      import; type(c_ptr), value :: cs; type(c_ptr), value :: ctx; character(kind=c_char) :: msg(*) 
      integer(c_int), value :: msg_len
    end function
    integer(c_int) function temf_case_write(cs, ctx, root, msg, msg_len) bind(C, name="temf_case_write")
      import; type(c_ptr), value :: cs; type(c_ptr), value :: ctx; character(kind=c_char) :: root(*) 
      character(kind=c_char) :: msg(*); integer(c_int), value :: msg_len
    end function
    integer(c_int) function temf_case_run(root, device, flags, msg, msg_len) bind(C, name="temf_case_run")
      import; character(kind=c_char) :: root(*); integer(c_int), value :: device; integer(c_int), value :: flags 
      character(kind=c_char) :: msg(*); integer(c_int), value :: msg_len
    end function
  end interface
end module temf_b200
