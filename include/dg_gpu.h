/* dg_gpu.h — C ABI of the B200 explicit DG operator for the 3D compressible Euler equations on
 * affine tetrahedra (modal basis P0..P5, Lax-Friedrichs or Roe flux, SSP-RK3).
 *
 * It replaces the reference's explicit convection path:
 *   ExplicitConvection<Order, Flux, QuadC, QuadF>::eval(mesh, U, t)
 *       include/DG/DG_Schemes/ExplicitConvection.h:31-33, src/DG/DG_Schemes/ExplicitConvection.cpp:136-141
 *   its parts eval_cells / eval_internals / eval_boundarys   ExplicitConvection.h:34-44
 *   the drivers' explicit time loop  U += dt * (-(1/b) * eval(U))   examples/Vortex/123/VortexRK.cpp:264-271
 *   the drivers' diagonal mass b     examples/Eular1D/Sod1D/Riemann1D.cpp:108-121
 *
 * Conventions shared with the reference:
 *   - state and residual: element-major, basis-major, variable-minor, coef[e][5*b + k] with
 *     k in {rho, rho u, rho v, rho w, rho E} (include/Matrix/LongVector.h:10). Host buffers may
 *     have a padded element stride (LongVector pads each block to 32 bytes, DenseMatrix.h:15):
 *     pass it as elem_stride_bytes, or 0 for the packed 5*Nb*8 bytes.
 *   - residual sign and scaling are those of ExplicitConvection::eval: no mass inverse, no dt.
 *   - face_cells[f][1] == DG_NO_CELL marks a boundary face (uInt(-1) in ComputingMesh.h:21).
 *
 * All entry points return DG_OK (0) or a negative DG_E* code; nothing throws across the ABI.
 * A dg_ctx owns its device buffers; host pointers are borrowed for the duration of a call.
 * A dg_ctx is not safe for concurrent use from several host threads.
 */
#ifndef FVEDG_DG_GPU_H
#define FVEDG_DG_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DG_NO_CELL (-1)

enum dg_status {
    DG_OK = 0,
    DG_E_ARG = -1,        /* bad argument (null pointer, unsupported order or rule, ...) */
    DG_E_MESH = -2,       /* malformed mesh: bad index, face/cell mismatch, bad face map */
    DG_E_CUDA = -3,       /* a CUDA runtime call failed */
    DG_E_NOMEM = -4,      /* device or host allocation failed */
    DG_E_NONPHYSICAL = -5,/* the state has NaN/Inf or non-positive density or pressure */
    DG_E_WATCHDOG = -6,   /* a bounded device wait ran out (batched persistent form) */
    DG_E_STATE = -7,      /* call out of order (e.g. stepping before a state was set) */
    DG_E_IO = -8          /* file could not be opened, read or written, or failed its checksum */
};

enum dg_flux_kind { DG_FLUX_LF = 0, DG_FLUX_ROE = 1 };
enum dg_precision { DG_PREC_FP64 = 0, DG_PREC_MIXED = 1 };

/* BoundaryType of include/Mesh/ComputingMesh.h:71-86. eval_boundarys acts on Dirichlet and
 * Pseudo3DZ only; every other type contributes nothing (ExplicitConvection.cpp:47-125). */
enum dg_boundary {
    DG_BC_DIRICHLET = 0, DG_BC_NEUMANN = 1, DG_BC_ROBIN = 2, DG_BC_PSEUDO3DX = 3,
    DG_BC_PSEUDO3DY = 4, DG_BC_PSEUDO3DZ = 5, DG_BC_INFLOW = 6, DG_BC_OUTFLOW = 7,
    DG_BC_WALL = 8, DG_BC_WALLTD = 9, DG_BC_WALLTN = 10, DG_BC_WALLTR = 11
};

/* Quadrature rule ids. -1 selects the reference's AutoQuadSelector choice for the order
 * (include/GaussQuadrature/AutoQuadSelectorTet.h:2-50, AutoQuadSelectorTri.h:1-45). */
enum dg_tet_rule {
    DG_TET_D2P4 = 0, DG_TET_D4P11 = 1, DG_TET_D5P15 = 2, DG_TET_D6P23 = 3,
    DG_TET_D7P31 = 4, DG_TET_D8P44 = 5, DG_TET_D9P57 = 6, DG_TET_D11P94 = 7
};
enum dg_tri_rule { DG_TRI_D3P4 = 0, DG_TRI_D3P6 = 1, DG_TRI_D4P7 = 2, DG_TRI_D10P24 = 3, DG_TRI_D13P36 = 4 };

/* Flattened mesh. Topology follows DGMesh (include/Mesh/MeshGenerator.h:46-57) and
 * ComputingMesh(const DGMesh&) (src/Mesh/ComputingMesh.cpp:268-298); geometry follows
 * CompTetrahedron / CompTriangleFace (ComputingMesh.cpp:27-171).
 *
 * Two ways to describe it:
 *  (a) from a reference ComputingMesh: give face_cells, face_natural, face_normal, face_area,
 *      cell_invjac and cell_detj exactly as the reference holds them (m_neighbor_cells,
 *      m_natural_coords, m_normal, m_area, m_invJac, compute_jacobian_det());
 *  (b) from raw topology: leave the geometry pointers NULL and give points, cell_nodes,
 *      face_nodes (and, for periodic faces, face_nodes1 + face_periodic). The library then
 *      computes the geometry with the reference's formulas and operation order: connectivity,
 *      orientation and face maps bit for bit, normals, areas and J^-T to a few ulp (the two builds
 *      contract different a*b+c into FMAs). */
typedef struct dg_mesh_desc {
    int64_t ncell;
    int64_t nface;
    const int64_t* face_cells;   /* [nface][2]; [f][1] = DG_NO_CELL on a boundary face        */
    const uint8_t* face_bc;      /* [nface] dg_boundary for boundary faces; NULL = Pseudo3DZ   */
    /* (a) geometry as held by a reference ComputingMesh (all or none) */
    const double* face_natural;  /* [nface][2][3][3] m_natural_coords                          */
    const double* face_normal;   /* [nface][3] unit normal out of cells[0]                     */
    const double* face_area;     /* [nface]                                                    */
    const double* cell_invjac;   /* [ncell][9] row-major inverse of rows {p1-p0,p2-p0,p3-p0}   */
    const double* cell_detj;     /* [ncell] 6 |V|                                              */
    /* (b) raw topology */
    int64_t npts;
    const double* points;        /* [npts][3]                                                  */
    const int64_t* cell_nodes;   /* [ncell][4]                                                 */
    const int64_t* face_nodes;   /* [nface][3] (face node order defines the face parameters)   */
    const int64_t* face_nodes1;  /* [nface][3] the face's nodes as numbered in cells[1]; NULL = face_nodes */
    const uint8_t* face_periodic;/* [nface] 1 = periodic pair (normal by the boundary rule); NULL = none */
    /* Ghost elements (one mesh split across processes, fve_dg_b200/partition.py): the last nghost
     * cells are copies of elements that another process owns. A ghost needs only the faces it
     * shares with owned cells (1 to 4); the context holds its state and computes the fluxes of those
     * faces but no residual, limiting, viscous term or reduction for it: residual rows of ghosts are
     * left unwritten and dg_conservation / dg_max_wave_speed / dg_check_state cover owned cells.
     * The viscous penalty of a face uses its cells[0]'s volume over the areas of its four sides:
     * for a ghost with missing faces these come from its vertices (form (b)); in form (a) give the
     * viscous operator ghosts with all four faces. 0 for an ordinary mesh (zero-initialise the
     * struct). */
    int64_t nghost;
} dg_mesh_desc;

typedef struct dg_config {
    int order;       /* 0..5 (FP64 tensor-core kernels and the mixed-precision form: 1..4) */
    int flux;        /* dg_flux_kind */
    int quad_vol;    /* dg_tet_rule or -1 */
    int quad_face;   /* dg_tri_rule or -1 */
    double gamma;    /* 1.4 (AirFluxC) or 5/3 (MonatomicFluxC), any value > 1 accepted */
    int precision;   /* dg_precision */
    int device;      /* CUDA device ordinal */
    int schedule;    /* 0: two launches per RK stage (face fluxes, then elements);
                        1: one persistent launch per stage over a tile list of face and element
                           tiles interleaved by mesh region (mixed precision only; see dg_autotune) */
    int limiter;     /* 0: none; 1: positivity-preserving limiter after every RK stage, bounds from
                        the stage input's values at the volume points; 2: the same with bounds from
                        the neighbours' means (PositiveLimiter<.., OnlyNeigbAvg = true>); see dg_limit */
    double mu;       /* 0: Euler. > 0: compressible Navier-Stokes stepping: every SSP-RK3 stage adds the
                        viscous residual of dg_viscous_residual with this viscosity, L = (R_visc -
                        R_conv) / b as the reference's viscous driver (tests/test_diffusion.cpp:381-382) */
    double prandtl;  /* Prandtl number of that viscous term (> 0 when mu > 0) */
} dg_config;

typedef struct dg_ctx dg_ctx;

/* Create a context: validates and uploads the mesh, builds basis/face tables and the diagonal
 * mass. Replaces constructing ExplicitConvection<...> plus the driver's mass loop. */
dg_ctx* dg_create(const dg_mesh_desc* mesh, const dg_config* cfg, int* err);
void dg_destroy(dg_ctx* ctx);

/* Residual R(U) with the sign and scaling of ExplicitConvection::eval (ExplicitConvection.cpp:136-141),
 * host buffers in, host buffer out. part: 0 = eval, 1 = eval_cells, 2 = eval_internals,
 * 3 = eval_boundarys. */
int dg_residual(dg_ctx* ctx, const double* U, double* R, size_t elem_stride_bytes, double t, int part);

/* Same on device buffers (packed layout), enqueued on `stream` (a cudaStream_t, NULL = default). */
int dg_residual_device(dg_ctx* ctx, const double* U_dev, double* R_dev, double t, int part, void* stream);

/* Residual on device buffers that allocates nothing. This entry point has no counterpart in the
 * reference. It is for callers that cannot call cudaMalloc once they are running: applications and
 * frameworks that hand all device memory to their own pool allocator at start-up and forbid raw
 * cudaMalloc afterwards (a raw allocation there either fails, because the pool already holds the
 * memory, or takes memory the pool has counted as free), and time-critical loops that must not
 * allocate because cudaMalloc and cudaFree can synchronise the device. Such a caller creates the
 * context during its set-up and may then call this any number of times.
 * It computes what dg_residual_device computes with the FP64 kernels, but the face-flux scratch
 * (nface * nqf * 5 doubles) lives in one fixed device array of this library,
 * dg_static_scratch_capacity() doubles (32 MiB), that every GPU which loads the library holds
 * until the process exits. Meshes whose face fluxes do not fit are rejected with DG_E_ARG. On a
 * context created with DG_PREC_MIXED it still runs the FP64 kernels, so its result is the FP64
 * residual (what dg_residual_device returns on an FP64 context), not the mixed-precision one.
 * The first call on a device looks up that device's copy of the array (cudaGetSymbolAddress with
 * the context's device current) and keeps the address for the life of the process; make that first
 * call before any stream capture begins, and do not call this after cudaDeviceReset on that device.
 * Every call shares the one array and it keeps the last call's contents; nothing in it has to start
 * at zero (each call writes every entry it reads). Calls whose kernels overlap on the GPU (on
 * different streams, or from several contexts on one device) race on the array: serialise them. */
int dg_residual_device_static(dg_ctx* ctx, const double* U_dev, double* R_dev, int part, void* stream);
/* Capacity of that array, in doubles. */
int64_t dg_static_scratch_capacity(void);

/* Device-resident time stepping (the driver loop of VortexRK.cpp:264-271 with SSP-RK3). */
int dg_set_state(dg_ctx* ctx, const double* U, size_t elem_stride_bytes);
int dg_get_state(dg_ctx* ctx, double* U, size_t elem_stride_bytes);
int dg_ssprk3(dg_ctx* ctx, double dt, int nsteps);
/* Capture one SSP-RK3 step in a CUDA graph and replay it nsteps times. */
int dg_ssprk3_graph(dg_ctx* ctx, double dt, int nsteps);

/* Ensembles of independent solves on meshes of different sizes (new; the reference runs one mesh
 * per process). The meshes are laid end to end as one disconnected mesh in one context, all with
 * the same configuration; every stage of every instance then runs in the same launches.
 * dg_set_state / dg_get_state / dg_conservation act on the concatenated state, instance i owning
 * elements [offsets[i], offsets[i+1]). */
dg_ctx* dg_create_ensemble(const dg_mesh_desc* meshes, int ninstances, const dg_config* cfg, int* err);
/* Writes ninstances + 1 element offsets; returns ninstances (1 for an ordinary context). */
int dg_ensemble_offsets(const dg_ctx* ctx, int64_t* elem_offsets);
/* nsteps SSP-RK3 steps with a per-instance time step dt[ninstances]; use_graph replays one CUDA
 * graph per step (the dt values are read from device memory, so one graph serves any dt). */
int dg_ssprk3_ensemble(dg_ctx* ctx, const double* dt, int nsteps, int use_graph);

/* Autotuner of the mixed-precision form: times each candidate on the current state (restored
 * afterwards), keeps the fastest and writes a JSON record of every candidate and the choice into
 * report[len]. Persistent schedule: face and element groups per tile, CTAs per SM, mesh regions,
 * lag. Two-launch schedule: the element kernel's shape (elements per CTA and CTAs per SM, with its
 * loads issued phase by phase or each group's rows staged in shared memory by TMA bulk copies). */
int dg_autotune(dg_ctx* ctx, double dt, char* report, size_t len);
/* Pins the element-kernel shape of the two-launch mixed schedule (what dg_autotune chooses; this
 * replays a recorded choice without timing): staged = 0 issues the group's loads phase by phase,
 * staged = 1 stages each group's rows in shared memory by TMA bulk copies (orders 1..3) with
 * ctas_per_sm = 1 or 2 resident CTAs. Both shapes give bit-identical results. DG_E_ARG for other
 * values, an FP64 context or a staged shape at order 4. New: no reference counterpart. */
int dg_set_element_shape(dg_ctx* ctx, int staged, int ctas_per_sm);

/* Self-test of the failure detection of the batched persistent form (mixed precision, schedule 1):
 * runs stage 0 of one SSP-RK3 step with the completion count that face region 0 must reach raised
 * by one, so every wait of an element tile on that region runs out after `polls` polls (each about
 * 64 ns) instead of ending; the count is restored afterwards. Returns what the stage reports:
 * DG_E_WATCHDOG when the expired waits were recorded on the device and read back by the host. The
 * stage writes only U^(1), so U^n is unchanged and the context stays usable. New: the reference has
 * no device code and no such check. */
int dg_watchdog_selftest(dg_ctx* ctx, int64_t polls);

/* Same as dg_ssprk3, with CUDA events around every kernel launch on the context's stream.
 * out[2k] = total milliseconds and out[2k+1] = launch count of kernel class k < nclass:
 * 0 = face fluxes, 1 = element kernel (volume, face integrals, update), 2 = the persistent stage
 * kernel (mixed form, persistent schedule), 3 = viscous residual (Navier-Stokes stepping),
 * 4 = limiter. */
int dg_ssprk3_timed(dg_ctx* ctx, double dt, int nsteps, double* out, int nclass);
/* The context's CUDA stream (a cudaStream_t) on which every kernel of the context runs. */
void* dg_stream(dg_ctx* ctx);

/* One mesh across several GPUs (new; the reference runs one mesh in one process). Each process
 * creates a context on its part of the mesh, owned elements first and then ghost copies of the
 * neighbours that other processes own, and runs SSP-RK3 one stage at a time, filling the ghost rows
 * of the stage input from their owners in between (fve_dg_b200/partition.py).
 * State buffer `which` on the device, packed [ncell][5*Nb]: 0 = U^n, 1 = U^(1), 2 = U^(2); stage s
 * reads buffer s and writes buffer (s + 1) mod 3. NULL for a bad argument. */
double* dg_state_device(dg_ctx* ctx, int which);
/* After rows of state buffer `which` were written from outside the library (a halo exchange): kept
 * for drivers written against earlier versions, in which the mixed form held split copies of the
 * coefficients. Now every kernel splits the FP64 rows as it loads them, so there is nothing to
 * refresh: it checks its arguments and returns DG_OK. */
int dg_refresh_split(dg_ctx* ctx, int which, const int64_t* elems_dev, int64_t n, void* stream);
/* Enqueues stage `stage` (0, 1, 2) of one SSP-RK3 step, with the limiter when configured, on the
 * context's stream and returns; dg_ssprk3(ctx, dt, 0) waits for it and reports a watchdog error.
 * Run the stages of a step in order 0, 1, 2; between them, write only ghost rows from outside. */
int dg_ssprk3_stage(dg_ctx* ctx, double dt, int stage);
/* The same stage in two phases, so that a halo exchange overlaps work: phase 0 enqueues what reads
 * no ghost row (in the mixed two-launch form, the fluxes of the faces between owned elements;
 * otherwise nothing), phase 1 the rest. Between them, write the ghost rows of the stage input;
 * phases 0 then 1 launch exactly what dg_ssprk3_stage launches. */
int dg_ssprk3_stage_phase(dg_ctx* ctx, double dt, int stage, int phase);

/* One mesh split across processes, for drivers that exchange halos with MPI or NCCL themselves
 * (fve_dg_b200/partition.py is the Python form of the same plan). New: the reference runs one
 * mesh per process.
 * dg_partition_create: rank `rank`'s part under owner[ncell] (values 0..nparts-1) of a raw-topology
 * mesh (form (b), nghost = 0). Its local mesh holds the owned elements (ascending global id), then
 * the ghosts: face neighbours of owned elements that other ranks own (ascending). Its faces are the
 * global faces that touch an owned element, in global order and orientation, so an owned element's
 * residual equals its whole-mesh residual once the ghost rows hold their owners' values. The plan
 * sends to each peer q the rows of owned elements that are ghosts of q and receives from q the
 * ghosts q owns, both in ascending global order, so the lists of the two sides match. */
typedef struct dg_partition dg_partition;
dg_partition* dg_partition_create(const dg_mesh_desc* mesh, const int32_t* owner, int rank, int* err);
void dg_partition_destroy(dg_partition* part);
/* The local mesh as a descriptor for dg_create (nghost set; pointers into the plan, the points
 * shared with the global mesh's array), valid until dg_partition_destroy. */
int dg_partition_local_mesh(const dg_partition* part, dg_mesh_desc* local);
int dg_partition_counts(const dg_partition* part, int64_t* n_owned, int64_t* n_ghost, int* n_send_peers,
                        int* n_recv_peers);
/* Global element id of every local element [n_owned + n_ghost]; global face id of every local face. */
const int64_t* dg_partition_l2g(const dg_partition* part);
const int64_t* dg_partition_global_faces(const dg_partition* part);
/* Peer i (ascending rank) to send to / receive from: its rank, the row count and the local rows. */
int dg_partition_send(const dg_partition* part, int i, int* peer, int64_t* n, const int64_t** rows);
int dg_partition_recv(const dg_partition* part, int i, int* peer, int64_t* n, const int64_t** rows);
/* Device gather / scatter of whole element rows (5 Nb doubles) of state buffer `which` (as
 * dg_state_device) for the exchange, on `stream` (0 = the context's stream): pack copies row
 * rows_dev[i] to slot i of buf_dev, unpack copies slot i into row rows_dev[i]. Rows outside the
 * context's cells are skipped. */
int dg_halo_pack(dg_ctx* ctx, int which, const int64_t* rows_dev, int64_t n, double* buf_dev, void* stream);
int dg_halo_unpack(dg_ctx* ctx, int which, const int64_t* rows_dev, int64_t n, const double* buf_dev, void* stream);

/* Explicit viscous operator, replaces ExplicitDiffusion<Order, QuadC, QuadF>::eval(mesh, U, t)
 * (include/DG/DG_Schemes/ExplicitDiffusion.h:133-626) with the context's order and rules: the
 * interior-penalty Navier-Stokes viscous residual R of U, same sign and scaling as the reference
 * (volume term subtracted, face terms added on cells[0] and subtracted on cells[1]). The reference
 * fixes mu = 1 and Pr = 1; here they are arguments (gamma is the context's). Dirichlet faces use the
 * data of dg_set_dirichlet. Host buffers with the element stride of dg_residual. */
int dg_viscous_residual(dg_ctx* ctx, const double* U, double* R, size_t elem_stride_bytes, double mu, double prandtl);
/* Same on device buffers, enqueued on `stream` (a cudaStream_t, 0 = default). The first call on a
 * context allocates the operator's per-face buffer (nface * (5 nqf + Nb) doubles) and its tables (a
 * context with dg_config.mu > 0 has them from its creation); calls on one context share that buffer,
 * so calls whose kernels could overlap, and Navier-Stokes steps of the same context, must be
 * serialised with them. */
int dg_viscous_residual_device(dg_ctx* ctx, const double* U_dev, double* R_dev, double mu, double prandtl,
                               void* stream);

/* Positivity-preserving limiter, replaces PositiveLimiter<P, QuadC, OnlyNeigbAvg>::constructMinMax
 * (current, previous) followed by apply(current, previous) (include/DG/DG_Schemes/PositiveLimiter.h:
 * 12-261, called so in examples/Eular1D/Sod1D/Riemann1D.cpp:194-195), with QuadC the context's volume
 * rule: bounds from Uprev, the three limiting steps on U in place. Element means are unchanged.
 * Host buffers with the element stride of dg_residual. only_neighbor_avg selects OnlyNeigbAvg. */
int dg_limit(dg_ctx* ctx, double* U, const double* Uprev, size_t elem_stride_bytes, int only_neighbor_avg);
/* Same on device buffers (packed [ncell][5*Nb]), enqueued on `stream` (a cudaStream_t, 0 = default). */
int dg_limit_device(dg_ctx* ctx, double* U_dev, const double* Uprev_dev, int only_neighbor_avg, void* stream);

/* Binary checkpoint / restart of the device state (new: the reference writes text solution files,
 * examples/Eular1D/Sod1D/Riemann1D.cpp:249-286, which fve_dg_b200/io.py reads and writes). The file
 * holds a header (order, rules, flux, precision, mesh sizes, gamma, time t, step), U^n in FP64 and a
 * checksum. Loading checks that the context has the same order, volume rule and mesh sizes
 * (DG_E_MESH otherwise) and the checksum (DG_E_IO), then sets the state; t and step may be NULL. */
int dg_save_checkpoint(dg_ctx* ctx, const char* path, double t, int64_t step);
int dg_load_checkpoint(dg_ctx* ctx, const char* path, double* t, int64_t* step);

/* Diagonal mass b[e][5i+k] = detJ * sum_g w_g phi_i(x_g)^2 (Riemann1D.cpp:108-121). */
int dg_mass(dg_ctx* ctx, double* mass, size_t elem_stride_bytes);

/* Boundary data: U_D at every face point of every Dirichlet face, [nface][nqf][5] indexed by face
 * id (entries of other faces are ignored). Stands in for the rho_Xi .. rhoe_Xi hooks of
 * include/base/exact.h:32-52 evaluated at the face points (ExplicitConvection.cpp:47-53). */
int dg_set_dirichlet(dg_ctx* ctx, const double* UD);

/* Conservation sums of the device state (new; the reference drivers have none):
 * out[0..4] = integrals of rho, rho u, rho v, rho w, rho E; out[5] = integral of rho|u|^2/2. */
int dg_conservation(dg_ctx* ctx, double out[6]);

/* Largest LF wave speed |u| + c over the volume points of the device state (for a CFL dt). */
int dg_max_wave_speed(dg_ctx* ctx, double* lam);

/* Non-physical-state check of the device state: returns DG_OK or DG_E_NONPHYSICAL and writes the
 * number of offending volume points. */
int dg_check_state(dg_ctx* ctx, int64_t* bad_points);

/* Sizes and the rules actually used. */
int dg_info(const dg_ctx* ctx, int* num_basis, int* nq_vol, int* nq_face, int* quad_vol, int* quad_face);

/* Geometry as the reference's ComputingMesh computes it from raw topology (form (b) of
 * dg_mesh_desc): unit normals, areas, natural coordinates [nface][2][3][3], J^{-T} [ncell][9],
 * detJ, centroids. Host-only; no device needed. */
int dg_mesh_geometry(const dg_mesh_desc* mesh, double* normal, double* area, double* natural,
                     double* invjac, double* detj, double* centroid);

/* Face maps: for every face and side the code 0..23 of the ordered vertex triple
 * (slot of face node 0, 1, 2 in the cell), derived from the natural coordinates; -1 for the
 * missing side of a boundary face. Host-only. */
int dg_face_perms(const dg_mesh_desc* mesh, int8_t* perm);

/* Basis values [npts][Nb] and reference gradients [npts][Nb][3] at reference-tet points
 * (DGBasisEvaluator<P>::eval_all / grad_all, include/DG/DG_Basis/DG_Basis_Evaluator.h:14-31). */
int dg_basis(int order, int npts, const double* xyz, double* phi, double* grad);
/* Quadrature rule: kind 0 = tet (points [n][3]), 1 = triangle (points [n][2]); weights [n].
 * Returns the number of points (either output may be NULL), or DG_E_ARG. */
int dg_quad_rule(int kind, int id, double* pts, double* w);
/* The reference's AutoQuadSelector choices for an order. */
int dg_auto_rules(int order, int* quad_vol, int* quad_face);

const char* dg_status_string(int status);
/* Name of the CUDA error behind the most recent DG_E_CUDA of this process (cudaGetErrorName), or
 * "cudaSuccess" if there was none. */
const char* dg_last_cuda_error(void);

/* Device name of the active context's GPU and the number of CUDA kernel launches issued by this
 * library since load (for launch accounting in benchmarks). */
int64_t dg_launch_count(void);

/* ---------------------------------------------------------------------------------------------
 * Periodic box mesh generator (new: the reference's split_hex6_scan is not periodic-conforming).
 * n^3 cubes on [lo,hi]^3, each cut into 6 tetrahedra around the main diagonal (Kuhn split, which
 * is translation invariant), vertices strictly inside the box jittered by a seeded uniform
 * +-jitter*h. Axes flagged periodic pair their boundary faces (face_cells[1] = partner cell,
 * face_nodes1 = translated nodes, face_periodic = 1); other boundary faces get boundary type bc.
 * Output arrays follow dg_mesh_desc form (b). */
typedef struct dg_box_mesh dg_box_mesh;
dg_box_mesh* dg_box_mesh_create(int n, const double lo[3], const double hi[3], double jitter,
                                uint64_t seed, const int periodic[3], int bc, int* err);
void dg_box_mesh_destroy(dg_box_mesh* m);
/* Borrowed views valid until dg_box_mesh_destroy. */
int dg_box_mesh_view(const dg_box_mesh* m, dg_mesh_desc* desc, const int64_t** cell_faces,
                     const int64_t** cell_cells);

#ifdef __cplusplus
}
#endif
#endif
