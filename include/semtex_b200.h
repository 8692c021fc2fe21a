/*
 * semtex_b200 -- C ABI of the B200 spectral-element--Fourier hot path.
 *
 * The reference (Semtex) has no FFI; its boundary for this path is the C++
 * class API of Domain / Field / ModalMatrixSys / AuxField and integrate().
 * Each entry point below replaces one of those calls (file:line given in the
 * reference tree) with plain pointers and sizes.
 *
 * Conventions
 *  - Every call returns 0 on success or a STX_E* code; stx_last_error()
 *    gives the message of the last failure on the calling thread.  (The
 *    reference prints and exits instead: veclib/util.c:24-46.)
 *  - Field data use the reference plane layout:
 *      data[k*plane_size + e*np*np + i*np + j]
 *    (src/auxfield.cpp:45-68); in Fourier space plane 0 = Re mode 0,
 *    plane 1 = Nyquist, planes 2m, 2m+1 = Re, Im of mode m.
 *  - Pointers named d_* are device pointers on the context's device; h_*
 *    are host pointers.  Device work runs asynchronously on the context's
 *    stream unless the call says it synchronises.
 *  - One host thread per context at a time.
 */
#ifndef SEMTEX_B200_H
#define SEMTEX_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define STX_OK 0
#define STX_EINVAL 1       /* bad argument or shape                         */
#define STX_ESESSION 2     /* session file / token / mesh error             */
#define STX_ENUMERIC 3     /* matrix not positive definite, singular hii    */
#define STX_ECUDA 4        /* CUDA runtime error                            */
#define STX_ENOCONV 5      /* PCG reached STEP_MAX (solution still written) */
#define STX_EUNSUPPORTED 6 /* feature outside this library's scope          */

#define STX_DIRECT 0 /* SolverKind DIRECT  (src/matrix.h:6-9) */
#define STX_JACPCG 1 /* SolverKind JACPCG                     */
/* DIRECT with the skeleton solve's packed inverses held in FP32 (sums in
 * FP64) and STX_REFINE (token, default 2; 0 = none, for error studies) FP64
 * iterative refinements of the skeleton solution, residuals from the FP64
 * element Schur complements.  Needs the two-level skeleton solve and a
 * non-singular system. */
#define STX_MIXED 2

#define STX_FORWARD 1  /* femlib/cfemdef.h FORWARD */
#define STX_INVERSE -1 /* femlib/cfemdef.h INVERSE */

typedef struct stx_context stx_context;
typedef struct stx_modal stx_modal;
typedef struct stx_dns stx_dns;
typedef struct stx_batch stx_batch;

/* Message of the last failed call on this thread ("" if none). */
const char* stx_last_error(void);

/* Read a FEML session, build mesh, geometry and numbering for every field,
 * upload them to `device`, work on `stream` (a cudaStream_t, or NULL for a
 * stream the context creates).  `overrides` holds "NAME=expr" token
 * assignments separated by ';' (or NULL).
 * Replaces the construction sequence FEML -> Mesh -> Geometry::set ->
 * Element -> BCmgr -> Domain (elliptic/drive.cpp:145-216,
 * dns/drive.cpp:157-248). */
int stx_context_create(const char* session_path, const char* overrides, int device,
                       void* stream, stx_context** out);
int stx_context_destroy(stx_context* ctx);

/* Geometry::nP/nZ/nElmt/planeSize (src/geometry.h:29-44). */
int stx_context_geometry(const stx_context* ctx, int* np, int* nz, int* nel, int* plane_size);
/* Field names as in <FIELDS>, NUL terminated, e.g. "uvwp" (Domain::field). */
int stx_context_fields(const stx_context* ctx, char* buf, int len);
/* Femlib::value (femlib/femlib.h:191-210) for a token or expression. */
int stx_token(const stx_context* ctx, const char* expr, double* value);
/* NumberSys sizes for a field (src/numbersys.h:44-46). */
int stx_numbering(const stx_context* ctx, char field, int* nglobal, int* nsolve, int* nband);
/* The `enumerate` utility (utility/enumerate.cpp:110-199) without a GPU:
 * reads the session and returns one field's numbering; nel and next =
 * 4*(np-1) give the sizes; h_btog / h_bmask (nel*next ints each,
 * boundary-major per element, or NULL) receive the
 * global numbers and the essential mask (the `.num` file's contents,
 * src/bcmgr.cpp:645-826).  Fields without essential nodes are numbered as
 * `enumerate -O3` numbers them (their singular k=0 system pins the highest
 * number); others by this library's reverse Cuthill--McKee. */
int stx_numbering_host(const char* session_path, const char* overrides, char field, int* nel,
                       int* next, int* nglobal, int* nsolve, int* nband, int* h_btog, int* h_bmask);
/* As stx_numbering_host, for Fourier mode `mode`: in cylindrical 3D sessions
 * with axis BCs <A> the numbering of modes 0, 1 and 2+ differ
 * (BCmgr::getNumberSys, src/bcmgr.cpp:550-583: the `.num` schemes u/U,
 * w/W, p/P, c/C); otherwise every mode takes the mode-0 numbering. */
int stx_numbering_host_mode(const char* session_path, const char* overrides, char field, int mode, int* nel,
                            int* next, int* nglobal, int* nsolve, int* nband, int* h_btog, int* h_bmask);
/* Elemental Helmholtz matrix of element `elmt` on the host, np^2 x np^2
 * row-major over the element's row-major nodes (Element::HelmholtzRow,
 * src/element.cpp:1411-1481; in cylindrical coordinates r-weighted, with
 * betak2 / r^2 + lambda2 as the Helmholtz constant).  *np (if not null)
 * receives N_P; h_matrix may be null. */
int stx_element_matrix_host(const char* session_path, const char* overrides, int elmt, double lambda2,
                            double betak2, int* np, double* h_matrix);
/* Element node locations, host buffers of nel*np*np (Element::_xmesh). */
int stx_mesh_coords(const stx_context* ctx, double* h_x, double* h_y);
/* Element mass weights (quadrature weight x Jacobian, Element::_Q4), host
 * buffer of nel*np*np. */
int stx_mesh_mass(const stx_context* ctx, double* h_q4);
/* Locate points in the mesh (HistoryPoint::locate, src/history.cpp:45-63,
 * over Element::locate, src/element.cpp:1061-1183, tokens TOL_POS and
 * NR_MAX): for each (xy[2i], xy[2i+1]) the first element whose Newton
 * iteration from its nearest node converges inside the element, in
 * h_elmt[i] (-1 when no element holds the point) with its canonical
 * coordinates (r, s) in h_rs[2i], h_rs[2i+1].  Host work, set-up. */
int stx_mesh_locate(const stx_context* ctx, int npts, const double* xy, int* h_elmt, double* h_rs);
/* The same from a session file, without a context or device. */
int stx_mesh_locate_host(const char* session_path, const char* overrides, int npts, const double* xy, int* h_elmt,
                         double* h_rs);
/* Relocate moved points (FluidParticle::integrate's search,
 * src/particle.cpp:155-175): for each point, Newton's iteration in its
 * element h_elmt[i] from its previous (r, s) in h_rs (Element::locate
 * without a guess); when that fails, or h_elmt[i] < 0, the search of
 * stx_mesh_locate.  h_elmt and h_rs are updated (-1 outside the mesh).
 * Host work. */
int stx_mesh_relocate(const stx_context* ctx, int npts, const double* xy, int* h_elmt, double* h_rs);
int stx_mesh_relocate_host(const char* session_path, const char* overrides, int npts, const double* xy,
                           int* h_elmt, double* h_rs);
/* Number of geometry families (elements sharing condensed matrices). */
int stx_mesh_families(const stx_context* ctx, int* nfamily);

/* AuxField = "function" (src/auxfield.cpp:198-220): evaluate an expression of
 * x, y, z, t and tokens at every node of every plane into host memory
 * h_out[nz*nel*np*np] (physical space, unpadded planes). */
int stx_field_evaluate(const stx_context* ctx, const char* expr, double t, double* h_out);

/* The expression evaluator on its own, host only (no device, no context):
 * `expr` of x, y, z, t evaluated at n points, with the default token table
 * (femlib/defaults.h:10-96) plus `assignments` ("NAME = expr" separated by
 * ';', or null).  compiled = 0: the interpreter (femlib/initial.y:138-249
 * restated); 1: the postfix program the device runs for forcing fields and
 * spatio-temporal forcing (dns/fieldforce.cpp:463-514), on the host.  *nops
 * (if not null) receives the program length after constant folding. */
int stx_expression_eval(const char* expr, const char* assignments, int compiled, int n, const double* x,
                        const double* y, const double* z, double t, double* out, int* nops);

/* FORCE-section token lookup, host only (FEML::valueFromSection on
 * <FORCE>, src/feml.cpp:519-560): the text after `token` on its line, up to
 * the next '=', into buf (len bytes, NUL-terminated).  *found = 0 when the
 * section or the token is absent. */
int stx_session_force_value(const char* session_path, const char* token, char* buf, int len, int* found);

/* Spectral vanishing viscosity operators, host only (SVV::operators and
 * SVV::coeffs / coeffs_z, src/svv.cpp:20-185): d_matrix[np*np] receives the
 * derivative matrix the viscous (lambda2 > 0) systems use -- the SVV one for
 * tokens SVV_EPSN = eps_n, SVV_MN = m_n, or the plain GLL derivative when SVV
 * is off -- and z_factors[(nz+1)/2] the factors of beta^2 k^2 of their Fourier
 * modes (SVV_EPSZ = eps_z, SVV_MZ = m_z); either pointer may be null. */
int stx_svv(int np, double eps_n, int m_n, int nz, double eps_z, int m_z, double kinvis, double* d_matrix,
            double* z_factors);

/* Evaluate a field's boundary values at time t in physical space on every
 * plane and Fourier-transform them (Field::evaluateBoundaries +
 * Field::bTransform, src/field.cpp:160-243).  Synchronises. */
int stx_field_bc_evaluate(stx_context* ctx, char field, double t);

/* ModalMatrixSys(lambda2, beta, base, nmodes, elmt, bsys, method)
 * (src/matrix.cpp:33-105): one condensed, Cholesky-factored (DIRECT) or
 * diagonally preconditioned (JACPCG) system per Fourier mode, with mode
 * constant (beta*k)^2.  Setup runs on the host cores in FP64 and uploads;
 * systems with equal constants and numbering are shared, as the reference's
 * MatrixSys cache shares them (src/matrix.cpp:85-97). */
int stx_modal_create(stx_context* ctx, char field, double lambda2, double beta, int base_mode,
                     int num_modes, int method, stx_modal** out);
int stx_modal_destroy(stx_modal* sys);
/* Band width and solve size of one mode (MatrixSys::_nband/_nsolve). */
int stx_modal_info(const stx_modal* sys, int mode, int* nsolve, int* nband);

/* Field::solve(f, MMS) (src/field.cpp:598-809) on device data: d_forcing is
 * the Fourier-space forcing (not modified), d_unknown receives the solution
 * (and holds the PCG initial guess on entry).  Uses the field's BC values
 * from the last stx_field_bc_evaluate.  For JACPCG, `tol_rel` and
 * `step_max` are TOL_REL / STEP_MAX; `iterations` (nz ints, may be NULL)
 * receives the per-plane iteration counts and the call synchronises.
 * A DIRECT solve is asynchronous and does not read the system's device
 * status word: after synchronising, stx_modal_status tells whether every
 * bounded wait of its kernels met its copy (else the solution is invalid). */
int stx_field_solve(stx_modal* sys, const double* d_forcing, double* d_unknown, double tol_rel,
                    int step_max, int* iterations);

/* Algorithmic bytes one DIRECT solve of this system must move, per phase of
 * stx_field_solve_profiled: bytes[4] = [element condensation, skeleton
 * solve (first half), skeleton solve (second half), element recovery].
 * Every matrix and field counted once. */
int stx_modal_bytes(const stx_modal* sys, double* bytes);

/* Kernel launches one stx_field_solve of a DIRECT system issues (two-level
 * systems split their modes into groups that run on parallel streams, each
 * group launching the whole sequence).  Instrumentation for benchmarks; no
 * counterpart in the reference. */
int stx_modal_launches(const stx_modal* sys, int* launches);

/* Field::solve for a DIRECT system with CUDA events recorded on the
 * context stream between its phases; synchronises and returns the device
 * milliseconds of [constrain+condense, forward band sweep, backward band
 * sweep, interior recovery] in phase_ms[4] and the number of kernel launches
 * in *launches (may be NULL).  Instrumentation for benchmarks. */
int stx_field_solve_profiled(stx_modal* sys, const double* d_forcing, double* d_unknown,
                             float* phase_ms, int* launches);

/* Field::solve for a DIRECT system that allocates no device memory.
 * No counterpart in the reference (which has no device memory at all).
 * For callers that cannot let a library call cudaMalloc after start-up --
 * hosts whose device memory is owned by their own allocator, or loops that
 * cannot take the synchronisation an allocation may imply.  The solve
 * scratch lives in a file-scope device array of 2^20 doubles (8 MiB);
 * problems needing more are rejected with STX_EINVAL.  The need is
 * 3 x nz x (nglobal rounded up to a multiple of 32) doubles for the two-level
 * skeleton solve, 2 x that for the single banded factor (token
 * STX_TWOLEVEL = 0).  CUDA loads the library's device code lazily, so the
 * array is mapped on a device by the first call made there, which looks up
 * its device address (cudaGetSymbolAddress): that first call may allocate
 * and synchronise like any module load and must be made at start-up, before
 * any stream capture; the device then holds the array until the process
 * exits, and later calls allocate nothing.  All calls on a device share the
 * one array and it keeps the last call's contents (the solve clears what it
 * accumulates into): calls that overlap on the GPU, e.g. issued on different
 * streams or contexts, race.  Asynchronous; the device status word is not
 * read (query stx_modal_status after synchronising).  Inputs, outputs and BC
 * values are as for stx_field_solve. */
int stx_field_solve_noalloc(stx_modal* sys, const double* d_forcing, double* d_unknown);

/* Synchronise and read the system's device status word: 0 when every
 * bounded wait of its solves met its copy; otherwise the solutions since the
 * word was set are not valid (1 banded sweep, 3 element kernels, 4 packed
 * skeleton products, 5 z-FFT).  Host-buffer solves check it themselves. */
int stx_modal_status(stx_modal* sys, int* status);

/* Field::solve for n fields at once, e.g. the velocity components of a
 * viscous substep (dns/integrate.cpp:186-193): solution i of systems[i] with
 * forcing d_forcing[i] (each field its own BC lines).  When the systems
 * share their matrices (equal constants and numbering: stx_modal_create
 * shares the storage) and n <= 3, one skeleton solve reads every matrix
 * tile once for all of them; otherwise the solves run one after another.
 * DIRECT (or MIXED, solved one by one) systems of one context. */
int stx_field_solve_multi(stx_modal* const* systems, int n, const double* const* d_forcing,
                          double* const* d_unknown);

/* AuxField::transform(sign) (src/auxfield.cpp:1157-1194) in place on nz
 * device planes of plane_size doubles. */
int stx_transform(stx_context* ctx, double* d_data, int sign);

/* Whole elliptic solve from host memory (elliptic/drive.cpp:61-96 with
 * elliptic/helmholtz.cpp:29-52): copy the physical-space forcing in, forward
 * transform, zero Nyquist, solve every mode, inverse transform, copy the
 * physical-space solution out.  Synchronises. */
int stx_elliptic_solve_host(stx_modal* sys, const double* h_forcing, double* h_solution);

/* n whole elliptic solves from host memory, as stx_elliptic_solve_host does
 * each, pipelined: the forcing of solve i + 1 is copied in and the solution
 * of solve i - 1 copied out while solve i runs (two device buffer sets, one
 * copy stream each way).  Host buffers should be pinned (cudaHostAlloc) for
 * the copies to overlap.  Synchronises; the device status words are read
 * once at the end.  No counterpart in the reference (one elliptic run is one
 * solve). */
int stx_elliptic_solve_host_batch(stx_modal* sys, int n, const double* const* h_forcing,
                                  double* const* h_solution);

/* The cudaStream_t all of the context's device work runs on. */
int stx_context_stream(const stx_context* ctx, void** stream);

/* ---- DNS time stepping: integrate() (dns/integrate.cpp:66-200) ----------
 * Velocity-correction splitting of order N_TIME with stiffly-stable /
 * extrapolation coefficients (src/integration.cpp:99-164), Cartesian
 * coordinates, fields "uvp" (2D) or "uvwp" (N_Z > 1).  advection selects the
 * nonlinear form as dns -S/-C/-N do (dns/drive.cpp:86-91): 0 skew-symmetric,
 * 1 alternating skew-symmetric (default), 2 convective, 3 Stokes.  Velocity
 * Helmholtz systems are DIRECT, with the reference's temporary JACPCG systems
 * for the first N_TIME-1 steps (dns/integrate.cpp:328-356).  Pressure BCs
 * may be <H> (high-order, computed each step: src/bcmgr.cpp:1036-1331).
 * Session token DEALIAS > 0 (with N_Z > 2) forms every nonlinear product on
 * the 3/2-padded z grid with AuxField::transform32's semantics
 * (src/auxfield.cpp:1197-1258), the reference's compile-time DEALIAS build
 * as a run-time token; by default products are not dealiased, as in the
 * reference's dns. */
int stx_dns_create(stx_context* ctx, int advection, stx_dns** out);
int stx_dns_destroy(stx_dns* dns);
/* Domain::restart semantics (src/domain.cpp:123-156): zero the multi-level
 * storage, step = 0, time = t0, re-evaluate BCs at t0. */
int stx_dns_restart(stx_dns* dns, double t0);
/* Set a field from physical-space host data [nz][nel*np*np], forward
 * transform, zero Nyquist (restart from a .rst file). */
int stx_dns_set_field(stx_dns* dns, char field, const double* h_phys);
/* Physical-space copy of a field (Domain::dump's INVERSE transform). */
int stx_dns_get_field(stx_dns* dns, char field, double* h_phys);
/* Take nsteps time steps (the while loop of integrate()).  Steady steps
 * (past the start-up orders, no time-dependent BCs) are captured once as a
 * CUDA graph of one cycle of steps -- from a storage-rotation and
 * alternating-form state back to it -- and replayed (token STX_DNS_GRAPH,
 * default 1; capture needs 12 steps left in the call). */
int stx_dns_advance(stx_dns* dns, int nsteps);
/* Running averages (Statistics, src/statistics.cpp; session token AVERAGE
 * 1: the raw fields, 2: also the velocity products A=uu B=uv C=vv D=uw E=vw
 * F=ww, 3: also the energy-equation correlations q d m n o r s t a b c
 * G-L).  stx_dns_stats_update is Statistics::update (the caller chooses
 * when: the dns program every IO_HIS steps).  stx_dns_stats_info returns the
 * averages' names in file order (NUL terminated) and the number of updates,
 * and sets that number when set_navg >= 0; get / set move one average in
 * physical space (set: Statistics::initialise from a .avg file). */
int stx_dns_stats_update(stx_dns* dns);
int stx_dns_stats_info(stx_dns* dns, char* names, int len, int* navg, int set_navg);
int stx_dns_stats_get(stx_dns* dns, char name, double* h_phys);
int stx_dns_stats_set(stx_dns* dns, char name, const double* h_phys);
/* Exchange the running averages with a second set of the same names (made,
 * zero, at the first call), with its own number of updates: the phase
 * averages (Statistics::phaseUpdate, src/statistics.cpp:587-611) are loaded
 * into it, updated and read out between two exchanges while the main
 * averages stay on the device unchanged. */
int stx_dns_stats_swap(stx_dns* dns);
/* stx_modal_status over every system of the time stepping (0: all valid). */
int stx_dns_status(stx_dns* dns, int* status);
/* Length of the captured step cycle (0: none) and the number of graph
 * launches so far. */
int stx_dns_graph_info(const stx_dns* dns, int* period, long long* launches);
int stx_dns_state(const stx_dns* dns, int* step, double* time);
/* Analyser (src/analysis.cpp:329-443), computed on the device from the
 * current (Fourier) velocity: modal energies per unit area
 * sum_i AuxField::mode_L2(m) over the DIM components (h_ek: (N_Z+1)/2
 * values); the divergence energy sum_m mode_L2(m) of div u, divided by
 * 2 pi / BETA; the CFL inverse time scale max(u.CFL(0), v.CFL(1)[, w.CFL(2)])
 * of Analyser::estimateCFL (CFL number = inv_dt * D_T). */
int stx_dns_modal_energy(stx_dns* dns, double* h_ek);
int stx_dns_divergence_energy(stx_dns* dns, double* value);
int stx_dns_cfl(stx_dns* dns, double* inv_dt);
/* History-point values (HistoryPoint::extract, src/history.cpp:66-78, over
 * AuxField::probe, src/auxfield.cpp:1621-1700), computed on the device from
 * the current (Fourier) fields: for points on elements h_elmt at (r, s) =
 * (h_rs[2i], h_rs[2i+1]) (from stx_mesh_locate) and z = h_z[i] (ignored with
 * fewer than 3 planes; null for z = 0), h_out[i * nfields + f] is the
 * physical-space value of field f, in FIELDS order. */
int stx_dns_probe(stx_dns* dns, int npts, const int* h_elmt, const double* h_rs, const double* h_z, double* h_out);
/* Forces on the edges of the boundary group named "wall" (DNSAnalyser::
 * analyse, dns/dnsanalysis.cpp:97-113: Field::normTraction and
 * tangTraction, src/field.cpp:392-458), from the mean (plane 0) fields on
 * the device: pressure[3] the pressure force, viscous[3] the viscous force
 * (-RHO KINVIS times the traction sums; z from the wall flux of w in 3D).
 * Zero without wall edges. */
int stx_dns_wall_forces(stx_dns* dns, double* pressure, double* viscous);
/* Tractions along the edges of the "wall" group, in physical space
 * (DNSAnalyser::analyse's session.wss data, dns/dnsanalysis.cpp:130-250:
 * Field::traction, src/field.cpp:533-593, per Fourier mode, then the inverse
 * z transform): *nline (if not null) receives N_P x the number of wall
 * edges; h_out (if not null; 3 x N_Z x nline doubles) receives the normal
 * (pressure), in-plane and out-of-plane viscous tractions, each as N_Z
 * planes of the wall lines, edges in the SURFACES section's order and
 * nodes along each side. */
int stx_dns_wall_traction(stx_dns* dns, int* nline, double* h_out);
/* Full-state checkpoint of the time stepping: the fields, the multi-level
 * velocity and nonlinear storage Us/Uf of every order (dns/integrate.cpp:
 * 99-136), the high-order pressure BC levels (BCmgr's _un / _hopbc,
 * src/bcmgr.cpp:951-993), the alternating form's switch, forcing state (SFD
 * filter, sponge mask) and running averages, with step and time.  The
 * reference's Domain::dump / restart (src/domain.cpp:123-215) keep the fields
 * only and restart at first order; a loaded checkpoint continues as the
 * uninterrupted run does (to round-off: the skeleton products sum with
 * atomics).  _size gives the bytes; _save fills a host buffer
 * (synchronises); _load restores one into a DNS of the same session
 * (re-evaluates BCs at the restored time; STX_EINVAL for a buffer of another
 * layout). */
int stx_dns_checkpoint_size(stx_dns* dns, unsigned long long* bytes);
int stx_dns_checkpoint_save(stx_dns* dns, void* h_buf, unsigned long long bytes);
int stx_dns_checkpoint_load(stx_dns* dns, const void* h_buf, unsigned long long bytes);
/* The ModalMatrixSys a steady step solves `field` with: the viscous system
 * of a velocity component (dns/integrate.cpp:186-193), the pressure system
 * (:244-252); owned by the DNS (not to be destroyed).  For stx_modal_bytes
 * and stx_modal_status. */
int stx_dns_system(stx_dns* dns, char field, stx_modal** sys);
/* Device pointer of a field's Fourier-space storage (nz x plane_size). */
int stx_dns_field_ptr(stx_dns* dns, char field, double** d_ptr);

/* ---- Discrete adjoint and tangent-linear model of the time step ---------
 * The reference has no derivative code; these differentiate the discrete
 * map its integrate() computes (dns/integrate.cpp:138-200): the velocity
 * given to stx_dns_set_field at the start of a recorded run -> the velocity
 * stx_dns_get_field reads at its end.  Checkpoints of the full state
 * (stx_dns_checkpoint_* blocks) are kept on the device every
 * `checkpoint_every` steps; the backward sweep recomputes one segment at a
 * time from its checkpoint and transposes its steps, so the memory is one
 * state per checkpoint plus one velocity per step of a segment.  The
 * transposed step reuses the step's symmetric condensed solves (with zero
 * BC data), transposes the projection, the high-order pressure BC terms
 * (src/bcmgr.cpp:1036-1331) and the z transforms, and linearises the
 * advection at the recorded velocity (dns/nonlinear.cpp:198-381).  Solves
 * that the forward run did by Jacobi-PCG (start-up orders, ITERATIVE) are
 * exact (DIRECT) in the derivatives.
 * Not differentiated (STX_EUNSUPPORTED at _create): DEALIAS, computed
 * outflow BCs, SVV, velocity-dependent forcing (sponge, drag, Coriolis,
 * SFD); other forcing and time-dependent BC values are data.
 * Host buffers of _backward and _tangent hold the velocity components one
 * after the other, each nz x nplane physical values as stx_dns_set_field
 * takes them.
 *   _record:   runs nsteps from the current state, keeping checkpoints;
 *   _backward: h_seed = d(objective)/d(final velocity) -> h_grad =
 *              d(objective)/d(initial velocity); the DNS is left at the
 *              end of the recorded run;
 *   _tangent:  h_dir (initial velocity direction) -> h_out, the derivative
 *              of the final velocity along it (the forward-mode check of
 *              _backward: <tangent(x), y> = <x, backward(y)>);
 *   _info:     first and last step of the record, checkpoint bytes. */
typedef struct stx_dns_adjoint stx_dns_adjoint;
int stx_dns_adjoint_create(stx_dns* dns, int checkpoint_every, stx_dns_adjoint** out);
int stx_dns_adjoint_destroy(stx_dns_adjoint* adj);
int stx_dns_adjoint_record(stx_dns_adjoint* adj, int nsteps);
int stx_dns_adjoint_backward(stx_dns_adjoint* adj, const double* h_seed, double* h_grad);
int stx_dns_adjoint_tangent(stx_dns_adjoint* adj, const double* h_dir, double* h_out);
int stx_dns_adjoint_info(const stx_dns_adjoint* adj, int* first_step, int* last_step,
                         unsigned long long* checkpoint_bytes);

/* ---- Batches of independent solves --------------------------------------
 * The reference solves one problem per `elliptic` run (elliptic/drive.cpp:
 * 61-96: one Field::solve).  stx_batch_create captures n DIRECT (or MIXED)
 * solves --
 * stx_field_solve(systems[i], d_forcing[i], d_unknown[i]) each on its own
 * context's stream -- as one CUDA graph whose independent problems are
 * parallel branches; it runs every solve once first, outside the capture
 * (the d_unknown buffers are written).  The device buffers are fixed in the
 * graph.  stx_batch_launch replays all n solves with one graph launch on
 * `stream` (NULL: a stream the batch creates; stx_batch_info returns it).
 * Systems may come from different contexts (different meshes and orders) on
 * one device; the systems and buffers must outlive the batch. */
int stx_batch_create(stx_modal* const* systems, const double* const* d_forcing, double* const* d_unknown,
                     int n, void* stream, stx_batch** out);
int stx_batch_launch(stx_batch* batch);
/* Number of systems, kernel launches per replay and the replay stream. */
int stx_batch_info(const stx_batch* batch, int* nsystems, int* kernel_nodes, void** stream);
int stx_batch_destroy(stx_batch* batch);

/* Synchronise the context's stream. */
int stx_sync(stx_context* ctx);

/* Device scratch the context owns: returns a device pointer to at least
 * `bytes` bytes (grown on demand; freed with the context). */
int stx_context_scratch(stx_context* ctx, unsigned long long bytes, void** d_ptr);

#ifdef __cplusplus
}
#endif

#endif /* SEMTEX_B200_H */
