/* zephyr_gpu.h -- C ABI of the B200 finite-volume step.
 *
 * The library replaces, on one GPU, the hot path of zephyr's single-material
 * solver: SmFluid::update (math/solver/sm_fluid.cpp:81-102) with its CFL time
 * step, fluxes, gradients, predictor and corrector, plus SmFluid::set_flags
 * (sm_fluid.cpp:517-559).  Paths in the comments are relative to the zephyr
 * source tree.
 *
 * Conventions
 *   - Every call returns 0 on success and a negative ZG_ERR_* code on failure;
 *     zg_last_error() then gives a message.  No C++ exception crosses the ABI.
 *   - A context owns one mesh, one solver configuration and all device memory
 *     for them, on the device it was created on.  Calls on one context must
 *     come from one host thread at a time (like SmFluid, the reference is not
 *     re-entrant either).
 *   - Host arrays are plain pointers; cell i of an array is element i, with
 *     the reference's cell numbering of a Rectangle mesh, ic = i * ny + j
 *     (mesh/euler/amr_cells_gen.cpp:145-151).
 *   - Work is queued on the context's stream; calls that return host data
 *     synchronise that stream.
 */
#ifndef ZEPHYR_GPU_H
#define ZEPHYR_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define ZG_OK 0
#define ZG_ERR_ARG (-1)     /* invalid argument or size */
#define ZG_ERR_CUDA (-2)    /* a CUDA call failed */
#define ZG_ERR_STATE (-3)   /* call out of order (no mesh, no configuration) */
#define ZG_ERR_ALLOC (-4)   /* device memory allocation failed */
#define ZG_ERR_NUMERIC (-5) /* a non-finite flux or state was produced */
#define ZG_ERR_TOO_LARGE (-6) /* mesh larger than zg_rect_step_noalloc accepts */

/* Boundary flags; values of zephyr's `enum class Boundary`
 * (geom/boundary.h:9-16). */
enum zg_boundary {
    ZG_BC_INNER = 0,
    ZG_BC_WALL = 1,
    ZG_BC_ZOE = 2,
    ZG_BC_PERIODIC = 3
};

/* Numerical fluxes; values of zephyr's `enum class Fluxes`
 * (math/cfd/flux/num_flux.h:11-21).  All eight of NumFlux::create
 * (num_flux.cpp:6-35) are implemented.  GODUNOV (the exact Riemann solver of
 * math/solver/riemann.cpp; its rarefaction powers use CUDA's pow) and HLLC_LM
 * (its low-Mach factor uses CUDA's sin) agree with the reference to a few
 * ulps rather than bit for bit.  HLLC_M, HLLC_LM, CIR1 and CIR2 run with the
 * PARITY kernels only. */
enum zg_flux {
    ZG_FLUX_GODUNOV = 0,
    ZG_FLUX_RUSANOV = 1,
    ZG_FLUX_HLL = 2,
    ZG_FLUX_HLLC = 3,
    ZG_FLUX_HLLC_M = 4,
    ZG_FLUX_HLLC_LM = 5,
    ZG_FLUX_CIR1 = 6,
    ZG_FLUX_CIR2 = 7
};

/* Slope limiters of math/cfd/limiter.cxx:15-153 (binary forms). */
enum zg_limiter {
    ZG_LIM_NONE = 0,
    ZG_LIM_UNIT,
    ZG_LIM_MINMOD,
    ZG_LIM_MC,
    ZG_LIM_VANLEER,
    ZG_LIM_VANALBADA1,
    ZG_LIM_VANALBADA2,
    ZG_LIM_CHARM,
    ZG_LIM_HCUS,
    ZG_LIM_HQUICK,
    ZG_LIM_KOREN,
    ZG_LIM_SMART,
    ZG_LIM_SUPERBEE
};

/* Equations of state (phys/matter/eos/ideal_gas.cpp, stiffened_gas.cpp). */
enum zg_eos { ZG_EOS_IDEAL = 0, ZG_EOS_STIFFENED = 1 };

/* Second-order time integration.  PREDICTOR_CORRECTOR is the reference
 * scheme (sm_fluid.cpp:89-98); HEUN is an extension: Heun's two-stage
 * Runge-Kutta on the corrector's spatial operator. */
enum zg_scheme { ZG_SCHEME_PREDICTOR_CORRECTOR = 0, ZG_SCHEME_HEUN = 1 };

/* Arithmetic of the face loop.  FP64 is the drop-in form. */
enum zg_precision { ZG_FP64 = 0, ZG_MIXED = 1 };

/* Kernel family.  PARITY evaluates every face flux from both sides in the
 * reference's order of operations without fused multiply-adds (bit-exact with
 * the reference); FAST computes each face once and lets the compiler fuse.
 * On a rectangle, FAST runs each second-order stage with HLLC or HLL as ONE
 * kernel (gradients, predictor, faces and update of a tile in shared
 * memory); FAST_TWO_PASS keeps the earlier two kernels per stage (gradients
 * and predictor stored in HBM, then the face pass), for comparison.  The
 * other fluxes use the two-pass kernels in both FAST families. */
enum zg_kernels { ZG_KERNELS_PARITY = 0, ZG_KERNELS_FAST = 1, ZG_KERNELS_FAST_TWO_PASS = 2 };

/* Solver configuration: SmFluid(Eos::Ptr) plus its setters
 * (math/solver/sm_fluid.h:41-71; defaults sm_fluid.cpp:16-23). */
typedef struct zg_smf_params {
    int eos_kind;    /* zg_eos */
    double gamma;    /* adiabatic index */
    double P0;       /* stiffened-gas pressure constant (0 for ideal gas) */
    double e0;       /* stiffened-gas energy constant (0 for ideal gas) */
    int flux;        /* zg_flux; SmFluid::set_method */
    int limiter;     /* zg_limiter; SmFluid::set_limiter */
    int accuracy;    /* 1 or 2, clamped like SmFluid::set_accuracy */
    int scheme;      /* zg_scheme */
    int precision;   /* zg_precision */
    int kernels;     /* zg_kernels */
    double CFL;      /* clamped to [0, 1] like SmFluid::set_CFL */
    double max_dt;   /* SmFluid::set_max_dt */
} zg_smf_params;

typedef struct zg_ctx zg_ctx;

/* Fill `p` with SmFluid's constructor defaults (sm_fluid.cpp:16-23):
 * HLLC, MC limiter, CFL 0.5, first order, no dt cap; ideal gas gamma 1.4. */
void zg_smf_default_params(zg_smf_params *p);

/* Map a limiter name to zg_limiter with the rules of Limiter(name)
 * (limiter.cxx:163-252); returns -1 for an unknown name. */
int zg_limiter_from_name(const char *name);

/* Create a context on CUDA device `device`. */
int zg_create(zg_ctx **out, int device);
int zg_destroy(zg_ctx *ctx);
const char *zg_last_error(const zg_ctx *ctx);

/* Use `stream` (a cudaStream_t) for all later work; NULL selects the
 * context's own stream. */
int zg_set_stream(zg_ctx *ctx, void *stream);

/* Build the mesh of Rectangle(x_min, x_max, y_min, y_max) with nx by ny
 * cells and boundary flags {left, right, bottom, top}; replaces
 * EuMesh(const Rectangle&) (mesh/euler/eu_mesh.cpp:70-102 ->
 * mesh/euler/amr_cells_gen.cpp:128-281).  PERIODIC on one side of an axis
 * makes both sides periodic (geom/generator/rectangle.cpp:182-189).  Any
 * previous state is discarded. */
int zg_mesh_rectangle(zg_ctx *ctx, int nx, int ny, double x_min, double x_max, double y_min,
                      double y_max, const int bounds[4]);
int zg_mesh_n_cells(const zg_ctx *ctx, int *n);

/* A mesh given cell by cell in the layout of zephyr's AmrCells / AmrFaces
 * (mesh/euler/amr_cells.h:49-104, amr_faces.h:83-154): every cell has 8 face
 * slots (slot k of cell i is entry 8*i + k); a slot holds a face or is
 * UNDEFINED (boundary flag -1) and is then skipped; a side shared with two
 * finer neighbours uses slots side and side + 4.  Cells are in the mesh's
 * storage order.  All arrays are host arrays. */
typedef struct zg_mesh_view {
    int n_cells;
    const double *center_x, *center_y; /* cell barycentres, n_cells each */
    const double *volume;              /* cell areas */
    const double *incircle;            /* incircle diameters (AmrCells::incircle_diameter) */
    const int *face_boundary;          /* 8 * n_cells: zephyr Boundary code, -1 = UNDEFINED */
    const int *face_neib;              /* 8 * n_cells: neighbour cell (the cell itself on boundaries) */
    const double *face_nx, *face_ny;   /* 8 * n_cells: outward normals */
    const double *face_cx, *face_cy;   /* 8 * n_cells: face centres */
    const double *face_area;           /* 8 * n_cells: face lengths */
} zg_mesh_view;

/* Load a mesh given cell by cell (for example a refined EuMesh); replaces
 * the EuMesh's AmrCells for the step.  Any previous state is discarded.  The
 * PARITY kernels run on such meshes; the FAST / MIXED kernels need a mesh from
 * zg_mesh_rectangle. */
int zg_mesh_upload(zg_ctx *ctx, const zg_mesh_view *mesh);

/* Axial symmetry (SmFluid::set_axial, sm_fluid.cpp:45-47, with a mesh made
 * by an axisymmetric generator, Rectangle::set_axial): y is the radius; the
 * fluxes are weighted by the faces' area_alt and the updates divided by the
 * cells' volume_alt (amr_cells_gen.cpp:267-279), and the radial momentum
 * gains the pressure source volume / volume_alt * p * dt (sm_fluid.cpp:
 * 160-170, 236-246, 341-350).  Host arrays: volume_alt (n_cells) and
 * face_area_alt (8 * n_cells, the slot order of zg_mesh_view); the centres
 * given to zg_mesh_upload are then the generator's axisymmetric barycentres.
 * NULL, NULL turns it off.  For a mesh from zg_mesh_upload, after each
 * upload; the PARITY kernels with first order or the predictor-corrector. */
int zg_mesh_set_axial(zg_ctx *ctx, const double *volume_alt, const double *face_area_alt);

/* ---- Adaptive mesh on the device ------------------------------------------
 * A rectangle mesh made adaptive keeps zephyr's AmrCells layout on the GPU
 * (9 map points, level, z-index and 8 face slots per cell) with room for
 * `capacity` cells.  The step then runs over the face slots with the PARITY
 * kernels (bit-exact) or the FAST kernels (FP64, face geometry derived from
 * each cell's centre and level), and zg_amr_refine adapts the mesh to the
 * cells' flags on the GPU.
 * Cell order, geometry, connectivity and distributed states match the
 * reference's EuMesh::refine on one rank bit for bit. */

/* State distributors of SmFluid::distributor(type) (sm_fluid.cpp:372-470). */
enum zg_distributor { ZG_DISTR_CONST = 0, ZG_DISTR_SLOPE = 1 };

/* Make the mesh of zg_mesh_rectangle adaptive with levels up to max_level
 * (clamped to [0, 15] like EuMesh::set_max_level, eu_mesh.cpp:178-184) and
 * device room for `capacity` cells; builds the base cells of
 * AmrCells(const Rectangle&) (amr_cells_gen.cpp:128-281).  Call before
 * zg_smf_configure.  Periodic boundaries are rejected: the reference's
 * EuMesh::init_amr fails on them ("Invalid rotation", mesh/amr/rotations.h).
 * The distributor starts as SLOPE, SmFluid::distributor's default type. */
int zg_amr_enable(zg_ctx *ctx, int max_level, int capacity);

/* EuMesh::set_distributor(solver.distributor(type)) (eu_mesh.cpp:194-196). */
int zg_amr_set_distributor(zg_ctx *ctx, int kind);

/* Set the adaptation flag of every cell from a host array of n_cells ints
 * (EuCell::set_flag).  zg_smf_set_flags writes the same flags on the device
 * (and may then be given a NULL host array); on an adaptive mesh it also
 * computes the limited gradients the SLOPE distributor uses, as
 * SmFluid::set_flags does (sm_fluid.cpp:517-522). */
int zg_amr_put_flags(zg_ctx *ctx, const int *flags);

/* Flags by the density-gradient criterion |grad rho| h / rho, h the square
 * root of the cell's volume: 1 above refine_above, -1 below coarsen_below, 0
 * between (no reference counterpart: the benchmark's AMR criterion, refine
 * above 0.05 and coarsen below 0.01), with the unlimited least-squares
 * density gradient.  The limited gradients of the current state are computed
 * too and kept for the SLOPE distributor, as zg_smf_set_flags keeps its own.
 * `flags` may be NULL (flags stay on the device). */
int zg_amr_set_flags_gradient(zg_ctx *ctx, double refine_above, double coarsen_below, int *flags);

/* Adapt the mesh to the flags; replaces EuMesh::refine (eu_mesh.cpp:290-359):
 * flag balancing, split and merge of cells with their hanging faces, the
 * distributor's states for new cells, compaction.  zg_mesh_n_cells gives the
 * new number of cells.  ZG_ERR_TOO_LARGE when the adaptation needs more than
 * `capacity` cells while it runs (the mesh is then unchanged; the flags are
 * balanced). Synchronises the stream. */
int zg_amr_refine(zg_ctx *ctx);

/* Counts of the last zg_amr_refine. */
typedef struct zg_amr_stats {
    int max_level, capacity;
    int n_before, n_after;   /* cells before / after */
    int n_coarse, n_refine;  /* cells merged into parents / split into children */
    int n_large;             /* cells held while the adaptation ran */
} zg_amr_stats;
int zg_amr_info(const zg_ctx *ctx, zg_amr_stats *out);

/* Host copies of the adaptive mesh's arrays; NULL members are skipped.
 * map_x, map_y: the 9 points of each cell's SqQuad map, point k of cell i at
 * 9 i + k with k = 3 (y + 1) + (x + 1) for the map coordinates x, y in
 * {-1, 0, 1}.  Face slots as in zg_mesh_view. */
typedef struct zg_amr_cells {
    double *center_x, *center_y, *volume, *incircle; /* n_cells each */
    double *map_x, *map_y;                           /* 9 * n_cells */
    int *level, *flag, *b_idx, *z_idx;               /* n_cells */
    int *face_boundary, *face_neib;                  /* 8 * n_cells */
    double *face_nx, *face_ny, *face_cx, *face_cy, *face_area; /* 8 * n_cells */
} zg_amr_cells;
int zg_amr_download(zg_ctx *ctx, const zg_amr_cells *out);

/* Configure the solver; replaces SmFluid(eos) and its setters.  The first
 * call allocates the solver's fields (SmFluid::add_types, sm_fluid.cpp:25-35)
 * with zero state and isolation counters; later calls only change the
 * parameters and keep the data, as the reference's setters do. */
int zg_smf_configure(zg_ctx *ctx, const zg_smf_params *p);
int zg_smf_set_max_dt(zg_ctx *ctx, double max_dt);

/* Copy the primitive state of every cell (the field `init`: density,
 * velocity x, velocity y, pressure, specific internal energy) from / to host
 * arrays of n_cells doubles each. */
int zg_state_upload(zg_ctx *ctx, const double *rho, const double *vx, const double *vy, const double *p,
                    const double *e);
int zg_state_download(zg_ctx *ctx, double *rho, double *vx, double *vy, double *p, double *e);

/* Isolation counters (the field `wait`, sm_fluid.cpp:354-364). */
int zg_wait_upload(zg_ctx *ctx, const int *wait);
int zg_wait_download(zg_ctx *ctx, int *wait);

/* One time step; replaces SmFluid::update (sm_fluid.cpp:81-102).
 * Asynchronous: the step's dt stays on the device until zg_smf_dt. */
int zg_smf_update(zg_ctx *ctx);

/* `n_steps` consecutive steps without host synchronisation (a driver's time
 * loop with a fixed max_dt). */
int zg_smf_update_n(zg_ctx *ctx, int n_steps);

/* dt of the last step; replaces SmFluid::dt() (sm_fluid.h:68).
 * Synchronises the stream. */
int zg_smf_dt(zg_ctx *ctx, double *dt);

/* Refinement flags of every cell into a host array of n_cells ints
 * (-1 coarsen, 0 keep, 1 refine); replaces the flag loop of
 * SmFluid::set_flags (sm_fluid.cpp:524-559). */
int zg_smf_set_flags(zg_ctx *ctx, int *flags);

/* Rows [row0, row0 + nrows) of a rectangle's FP64 state (rows along x:
 * cell (i, j) at i * ny + j), copied out (put = 0) or in (put = 1): fields
 * holds 5 blocks of nrows * ny doubles (density, vx, vy, pressure, energy),
 * wait the isolation counters of the same cells.  Host or device buffers.
 * The halo exchange of a slab decomposition (zephyr_b200/slabs.py) moves
 * these rows between ranks; it replaces the reference's mesh.sync of the
 * layers part.init and part.wait (sm_fluid.cpp:86-97). */
int zg_state_rows(zg_ctx *ctx, int row0, int nrows, double *fields, int *wait, int put);

/* The CFL quantity of the current state, min over cells of
 * incircle / (|v| + c), before CFL and max_dt (SmFluid::compute_dt,
 * sm_fluid.cpp:104-111), with the kernels the configured step uses.  A slab
 * decomposition takes the minimum over ranks (the reference's mpi::min) and
 * caps the next step with CFL times it (zg_smf_set_max_dt). */
int zg_smf_cfl_min(zg_ctx *ctx, double *dmin);

/* Limited gradients of the current state, SmFluid::compute_grad
 * (sm_fluid.cpp:116-125; gradient.h:226-282, 412-474), computed with the
 * bit-exact kernels and copied to host arrays of 4 * n_cells doubles each:
 * d_dx = [d rho/dx | d vx/dx | d vy/dx | d p/dx], d_dy likewise (field-major).
 * These are the d_dx / d_dy fields that SmFluid::set_flags leaves for the
 * slope distributor of the next EuMesh::refine (sm_fluid.cpp:404-458). */
int zg_smf_gradients(zg_ctx *ctx, double *d_dx, double *d_dy);

/* Number of kernels this context has launched (for launch accounting). */
int zg_launch_count(const zg_ctx *ctx, long long *count);

/* Kernel kinds reported by zg_kernel_times. */
enum zg_kernel_kind {
    ZG_K_DT = 0,      /* CFL minimum (SmFluid::compute_dt) */
    ZG_K_FLUX1,       /* first-order step (SmFluid::fluxes) */
    ZG_K_GRAD,        /* limited gradients (SmFluid::compute_grad) */
    ZG_K_STAGE1,      /* predictor (SmFluid::fluxes_stage1) */
    ZG_K_STAGE2,      /* corrector (SmFluid::fluxes_stage2) */
    ZG_K_HEUN_A,      /* Heun first stage */
    ZG_K_HEUN_B,      /* Heun second stage */
    ZG_K_FLAGS,       /* refinement flags */
    ZG_K_MM_DT,       /* multi-material CFL minimum (MmFluid::compute_dt) */
    ZG_K_MM_RECOVER,  /* PLIC reconstruction (MmFluid::interface_recovery) */
    ZG_K_MM_FLUX,     /* multi-material face loop, cells whose stencil is all pure (MmFluid::fluxes) */
    ZG_K_MM_CRP,      /* multi-material face loop, cells next to a mixed cell (composite Riemann fluxes) */
    ZG_K_MM_CLOSURE,  /* PT-equilibrium closure of updates that came out mixed (MixturePT::get_rPT) */
    ZG_K_TR_DT,       /* transport CFL minimum (Transfer::compute_dt) */
    ZG_K_TR_FLUX,     /* transport face fluxes, swept polygons or CRP (Transfer::fluxes_VOF / fluxes_CRP) */
    ZG_K_TR_UPDATE,   /* transport update of u1 */
    ZG_K_TR_NORMALS,  /* interface normals and sections (InterfaceRecovery compute_normals + find_sections) */
    ZG_K_TR_ADJUST,   /* one smoothing pass (InterfaceRecovery adjust_normals + find_sections) */
    ZG_K_MM_GRAD,     /* multi-material second order: limited gradients (MmFluid::compute_grad) */
    ZG_K_MM_STAGE1,   /* multi-material predictor (MmFluid::fluxes_stage1) */
    ZG_K_MM_STAGE2,   /* multi-material corrector (MmFluid::fluxes_stage2) */
    ZG_K_STEP,        /* fused predictor-corrector step of a rectangle (update in one kernel) */
    ZG_K_COUNT
};

/* Per-kernel device timing.  While enabled, every kernel launch is bracketed
 * by CUDA events on the context's stream.  zg_kernel_times synchronises the
 * stream, adds the elapsed times of all launches since the previous call into
 * ms[ZG_K_COUNT] and launches[ZG_K_COUNT] (either may be NULL), and resets. */
int zg_set_timing(zg_ctx *ctx, int on);
int zg_kernel_times(zg_ctx *ctx, double *ms, long long *launches);
const char *zg_kernel_name(int kind);

/* Wait for the context's stream. */
int zg_synchronize(zg_ctx *ctx);

/* ------------------------------------------------------------------------
 * Multi-material step: MmFluid (math/solver/mm_fluid.h:45-163), materials
 * in pressure and temperature equilibrium (MixturePT,
 * phys/matter/mixture_pt.h), first order, on a mesh from zg_mesh_rectangle.
 * The kernels are compiled for mixtures of two materials.
 * ------------------------------------------------------------------------ */

/* A material: IdealGas (kind ZG_EOS_IDEAL; P0, e0, T0 unused) or
 * StiffenedGas (ZG_EOS_STIFFENED), phys/matter/eos/ideal_gas.h,
 * stiffened_gas.h.  rho_ref is the reference density the mixture closure
 * starts from when no guess is given (Eos::density()). */
typedef struct zg_material {
    int kind;
    double gamma, P0, e0, Cv, T0, rho_ref;
} zg_material;

/* The named materials of IdealGas(name) (ideal_gas.cpp:14-24: "Air", "SF6")
 * and StiffenedGas(name) (stiffened_gas.cpp:13-86: "Air", "SF6", "Water",
 * "Water2", "Copper"/"Cu", "Lead"/"Pb", "Gas", "HeavyGas", "Liquid",
 * "Solid"), with the unit literals of phys/literals.h evaluated as the
 * reference evaluates them.  Returns ZG_ERR_ARG for an unknown name. */
int zg_material_named(int kind, const char *name, zg_material *out);

/* CRP mode: values of the reference's CrpMode (mm_fluid.h:31-41).  NONE
 * uses the plain mixture HLLC flux on every face; V3, V5, VS choose the
 * interface fraction by the heuristics of sections.cpp:50-84; PLIC
 * reconstructs the interface (the default).  MUSCL computes the limited
 * volume-fraction gradients of every cell each sub-step (fractions_grad,
 * mm_fluid.cpp:469-482; zg_mmf_grad_a reads them); the reference gives it no
 * face fraction (alpha_sigma returns NaN, mm_fluid.cpp:245-250, which
 * calc_crp_flux's assert rejects, mm_fluid.cpp:276), so a step that reaches
 * a composite face under MUSCL reports ZG_ERR_NUMERIC; faces whose states
 * are pure take the plain flux as in the reference. */
enum zg_crp_mode { ZG_CRP_NONE = 0, ZG_CRP_V3 = 1, ZG_CRP_V5 = 2, ZG_CRP_VS = 3, ZG_CRP_PLIC = 4, ZG_CRP_MUSCL = 5 };

/* MmFluid(MixturePT) and its setters (mm_fluid.h:58-100). */
/* Direction splitting of the multi-material step, values of DirSplit
 * (mm_fluid.h:28-32): NONE, one face loop over all faces; SIMPLE, the x faces
 * then the y faces, each with dt; STRANG, x faces with dt/2, y faces with dt,
 * x faces with dt/2 (mm_fluid.cpp:112-137). */
enum zg_dir_split { ZG_SPLIT_NONE = 0, ZG_SPLIT_SIMPLE = 1, ZG_SPLIT_STRANG = 2 };

typedef struct zg_mmf_params {
    int n_materials;          /* 2 */
    zg_material materials[4]; /* MixturePT{...}, in order */
    int crp_mode;             /* zg_crp_mode; set_crp_mode / set_method(CRP) */
    int accuracy;             /* 1 or 2 (set_accuracy) */
    double CFL;               /* clamped to [0, 1] (set_CFL) */
    double max_dt;            /* set_max_dt */
    int split;                /* zg_dir_split (set_splitting) */
    int precision;            /* zg_precision: FP64 (the reference's arithmetic) or MIXED (FP32 face
                                 states, wave speeds and HLLC fluxes of the pure faces: pure-stencil
                                 faces in first order, faces whose reconstructed states stay pure in
                                 second order (with a CRP mode); FP64 accumulation, update, EoS
                                 pressure recovery, reconstruction and its closures, composite
                                 Riemann fluxes, PLIC and dt) */
    int limiter;              /* zg_limiter of the second-order gradients (set_limiter; default MC) */
} zg_mmf_params;

/* MmFluid's constructor defaults (mm_fluid.cpp:16-26): CRP with PLIC,
 * CFL 0.7, first order, no dt cap; no materials. */
void zg_mmf_default_params(zg_mmf_params *p);

/* Configure the multi-material solver on the context's rectangle mesh;
 * replaces MmFluid(mixture), its setters and add_types (mm_fluid.cpp:28-40).
 * The first call allocates the fields; later calls keep the data. */
int zg_mmf_configure(zg_ctx *ctx, const zg_mmf_params *p);

/* Cell states as 14 doubles per cell: density, velocity x, velocity y,
 * pressure, specific internal energy, temperature, mass fractions [4], true
 * densities [4] (the fields of mmf::PState, math/cfd/models.h:167-180;
 * slots past n_materials hold fraction 0).  Host arrays. */
int zg_mmf_state_upload(zg_ctx *ctx, const double *cells);
int zg_mmf_state_download(zg_ctx *ctx, double *cells);

/* Initial states from density, velocity, pressure and mass fractions (4 per
 * cell), through the mixture closure as PState(density, velocity, pressure,
 * Fractions, mixture) does (models.cpp:180-188).  Host arrays. */
int zg_mmf_make_states(zg_ctx *ctx, const double *rho, const double *vx, const double *vy, const double *p,
                       const double *beta);

/* One time step; replaces MmFluid::update (mm_fluid.cpp:112-137).
 * Asynchronous; a state the reference would reject (negative density, a NaN
 * flux, the composite Riemann case it throws on) is reported as
 * ZG_ERR_NUMERIC by the next zg_mmf_dt or zg_mmf_state_download. */
int zg_mmf_update(zg_ctx *ctx);
int zg_mmf_update_n(zg_ctx *ctx, int n_steps);

/* dt of the last step (MmFluid::dt()); synchronises the stream. */
int zg_mmf_dt(zg_ctx *ctx, double *dt);

/* Refinement flags of MmFluid::set_flags (mm_fluid.cpp:836-885). */
int zg_mmf_set_flags(zg_ctx *ctx, int *flags);

/* CrpMode::MUSCL: the volume-fraction gradients of the last sub-step,
 * part.grad_a of MmFluid::fractions_grad (mm_fluid.cpp:469-482): per cell
 * 2 * n_materials doubles, (d alpha_i / dx, d alpha_i / dy) for each
 * material i.  ZG_ERR_STATE before a MUSCL step.  Synchronises the stream. */
int zg_mmf_grad_a(zg_ctx *ctx, double *out);

/* The PLIC reconstruction of the current state (interface_recovery,
 * mm_fluid.cpp:484-519): per cell and material the unit normal (x, y) and
 * the plane offset.  normals: 2 * n_materials doubles per cell; offsets:
 * n_materials per cell. */
int zg_mmf_interface(zg_ctx *ctx, double *normals, double *offsets);

/* ------------------------------------------------------------------------
 * Scalar VOF transport: zephyr's Transfer (math/solver/transfer.h:21-150)
 * advecting a volume fraction u1 with a prescribed velocity field, on the
 * context's rectangle mesh (non-periodic).  The velocity is the transfer
 * problem's field (problems/transfer.cpp:367-380), set in the parameters
 * instead of by overriding Transfer::velocity.
 * ------------------------------------------------------------------------ */

/* Transfer::Method values (transfer.h:25-51) with kernels: the CRP family,
 * VOF / VOF_CRP (swept-polygon fluxes with the PLIC reconstruction) and the
 * MUSCL family (compute_slopes and fluxes_MUSCL, transfer.cpp:345-469:
 * MUSCLd least-squares slopes, MUSCLn slopes from the interface planes,
 * MUSCL_MC limited slopes, and their CRP-limited forms) and WENO, WENO_CRP
 * (update_WENO, transfer.cpp:541-666: five-cell WENO stencils with the mesh's
 * periodic index wrap; at least 3 cells per axis). */
enum zg_tr_method {
    ZG_TR_CRP_V3 = 0, ZG_TR_CRP_V5 = 1, ZG_TR_CRP_SE = 2, ZG_TR_CRP_N1 = 3, ZG_TR_CRP_N2 = 4,
    ZG_TR_VOF = 5, ZG_TR_VOF_CRP = 6, ZG_TR_MUSCLD = 7, ZG_TR_MUSCLN = 8, ZG_TR_MUSCLD_CRP = 9,
    ZG_TR_MUSCLN_CRP = 10, ZG_TR_MUSCL_MC = 11, ZG_TR_MUSCL_MC_CRP = 12, ZG_TR_WENO = 13, ZG_TR_WENO_CRP = 14
};
enum zg_tr_velocity { ZG_TR_TRANSLATION = 0, ZG_TR_ROTATION = 1 };
/* Face directions of one update (mesh::Direction, amr_faces.h:75-80). */
enum zg_direction { ZG_DIR_ANY = 0, ZG_DIR_X = 1, ZG_DIR_Y = 2 };

typedef struct zg_tr_params {
    int method;      /* zg_tr_method (set_method) */
    double CFL;      /* clamped to [0, 1] (set_CFL) */
    int velocity;    /* zg_tr_velocity */
    double vel[3];   /* TRANSLATION: vx, vy; ROTATION: centre x, y and the angular velocity about z */
} zg_tr_params;

/* Transfer()'s defaults (transfer.cpp:44-49): VOF, CFL 0.5, and the base
 * class's velocity, the unit x translation (transfer.cpp:84-86). */
void zg_tr_default_params(zg_tr_params *p);

/* Configure on the context's rectangle (add_types, set_method, set_CFL);
 * the first call allocates the fields (u1 = 0), later calls keep them. */
int zg_tr_configure(zg_ctx *ctx, const zg_tr_params *p);

/* u1 per cell from a host array (u2 = 0); the interface is not rebuilt:
 * call zg_tr_update_interface as the reference's drivers do. */
int zg_tr_upload(zg_ctx *ctx, const double *u1);

/* u1 per cell; the interface normal n and base point p, (x, y) per cell;
 * any pointer may be NULL.  Host arrays; synchronises. */
int zg_tr_download(zg_ctx *ctx, double *u1, double *n, double *p);

/* Transfer::update_interface(mesh, smoothing) (transfer.cpp:656-658). */
int zg_tr_update_interface(zg_ctx *ctx, int smoothing);

/* Transfer::compute_dt (transfer.cpp:98-105): returns the CFL step (and
 * makes it the current dt, as the drivers then call set_dt with it). */
int zg_tr_compute_dt(zg_ctx *ctx, double *dt);
int zg_tr_set_dt(zg_ctx *ctx, double dt);
int zg_tr_get_dt(zg_ctx *ctx, double *dt);

/* Transfer::update(mesh, dir) (transfer.cpp:471-485): fluxes through the
 * faces of direction dir, the update of u1 and the reconstruction (three
 * smoothing passes for VOF, none for CRP). */
int zg_tr_update(zg_ctx *ctx, int dir);

/* `steps` iterations of the transfer problem's time loop
 * (problems/transfer.cpp:213-236) without leaving the device: dt from
 * compute_dt, clipped so that the time *time ends at t_end at most, then
 * update(X) and update(Y) when `split`, else update(ANY); *time is read
 * before and written after.  Asynchronous apart from the time copies. */
int zg_tr_advance(zg_ctx *ctx, int steps, int split, double t_end, double *time);

/* Transfer::set_flags (transfer.cpp:660-680): 1 where a neighbour's u1
 * differs, else -1.  Host array. */
int zg_tr_set_flags(zg_ctx *ctx, int *flags);

/* ------------------------------------------------------------------------
 * Output: VTU files and PVD series in zephyr's format (io/vtu_file.cpp,
 * io/pvd_file.cpp): XML header plus raw appended binary, cells written as
 * quadrilaterals (VtuStructure::fill_adaptive_hex_2D, vtu_file.cpp:186-201).
 * The arrays are packed from the device buffers on the GPU and written in
 * one pass; the bytes equal the reference writer's for the same mesh and
 * variables.  Meshes: zg_mesh_rectangle meshes and adaptive ones.
 * ------------------------------------------------------------------------ */

/* Sources of cell variables. */
enum zg_out_source {
    /* io::Variable's named variables (io/variable.cpp:11-160): */
    ZG_OUT_LEVEL = 0,   /* Int8 */
    ZG_OUT_INDEX = 1,   /* Int32, the cell's index */
    ZG_OUT_RANK = 2,    /* Int32, 0 */
    ZG_OUT_FLAG = 3,    /* Int8, the last refinement flags (0 before any) */
    ZG_OUT_B_IDX = 4,   /* Int32 */
    ZG_OUT_Z_IDX = 5,   /* Int32 */
    ZG_OUT_CENTER = 6,  /* Float32 x 3 */
    /* Float64 fields of the device state (`component` selects): */
    ZG_OUT_SMF = 7,     /* SmFluid: 0 density, 1 velocity x, 2 velocity y, 3 pressure, 4 energy */
    ZG_OUT_MMF = 8,     /* MmFluid: 0 density, 1 vx, 2 vy, 3 pressure, 4 energy, 5 temperature,
                           6 + k mass fraction k, 6 + n_materials + k true density k */
    ZG_OUT_TR = 9,      /* Transfer: 0 u1, 1 n.x, 2 n.y, 3 p.x, 4 p.y; 5 n and 6 p as 3-vectors (z = 0) */
    ZG_OUT_HOST = 10    /* Float64, a host array of n_cells values (any quantity the caller computes) */
};

typedef struct zg_out_var {
    const char *name;    /* the DataArray's Name */
    int source;          /* zg_out_source */
    int component;       /* field of ZG_OUT_SMF / MMF / TR */
    const double *host;  /* ZG_OUT_HOST: n_cells doubles */
} zg_out_var;

/* VtuFile::save(filename, mesh, variables) (vtu_file.cpp:555-584): creates
 * the parent directories and writes the file.  Synchronises. */
int zg_vtu_write(zg_ctx *ctx, const char *filename, const zg_out_var *vars, int n_vars);

/* PvdFile (pvd_file.h:12-89): open(filename, directory) writes the empty
 * collection (directory relative to the working directory, created if
 * missing); save writes `<directory>/<filename>_<k>.vtu` and adds it to the
 * collection at `timestep`. */
typedef struct zg_pvd zg_pvd;
int zg_pvd_open(zg_pvd **out, const char *filename, const char *directory);
int zg_pvd_save(zg_pvd *pvd, zg_ctx *ctx, const zg_out_var *vars, int n_vars, double timestep);
int zg_pvd_close(zg_pvd *pvd);

/* ------------------------------------------------------------------------
 * Adjoint mode (no counterpart in the reference): the gradient of
 *   J = mean pressure over the cells whose centre lies in a probe box
 * after `steps` Heun steps at a fixed dt, with respect to the initial density
 * field and the adiabatic index, by a discrete adjoint (reverse sweep) with
 * checkpoints every `checkpoint_every` steps.  The differentiated step: Heun's
 * method on the finite-volume operator of the second-order step (limited
 * least-squares slopes with a smooth van Albada limiter
 * phi(a, b) = (a (a + b) + eps) / (a^2 + b^2 + eps), HLLC with Davis wave
 * speeds, ideal gas), on a uniform rectangle periodic on both axes.  HLLC
 * branches are differentiated on the side the forward takes.
 * ------------------------------------------------------------------------ */
typedef struct zg_adj zg_adj;
typedef struct zg_adj_params {
    double gamma;          /* adiabatic index */
    double dt;             /* fixed time step (zg_adj_cfl_dt gives the CFL one) */
    int steps;             /* Heun steps */
    int checkpoint_every;  /* steps between stored states */
    double limiter_eps;    /* eps of the smooth limiter (default 1e-8) */
    double probe[4];       /* x_min, x_max, y_min, y_max of the probe box */
    int precision;         /* zg_precision: FP64, or MIXED (an FP64 primal step with FP32
                              slopes from FP64 neighbour differences; a reverse sweep with the
                              slopes' partials, face states, HLLC reverse and face cotangents
                              in FP32 and the adjoint states, their sums, the primitive map
                              and gamma in FP64) */
} zg_adj_params;

/* gamma 1.4, 100 steps, checkpoints every 10, eps 1e-8, probe [0.6,0.7]^2. */
void zg_adj_default_params(zg_adj_params *p);
int zg_adj_create(zg_adj **out, int device, int nx, int ny, double x_min, double x_max, double y_min,
                  double y_max);
int zg_adj_destroy(zg_adj *a);
const char *zg_adj_last_error(const zg_adj *a);
int zg_adj_set_stream(zg_adj *a, void *stream);
int zg_adj_launch_count(const zg_adj *a, long long *count);
/* dt = CFL min(hx, hy) / (|v| + c) over the cells (SmFluid::compute_dt on a
 * rectangle) for the given initial state (device arrays). */
int zg_adj_cfl_dt(zg_adj *a, double gamma, double CFL, const double *rho, const double *u, const double *v,
                  const double *p, double *dt);
/* J of the run from the initial state (rho, u, v, p: device arrays of
 * nx * ny doubles, cell (i, j) at i * ny + j); J on the host. */
int zg_adj_forward(zg_adj *a, const zg_adj_params *prm, const double *rho, const double *u, const double *v,
                   const double *p, double *J);
/* J, dJ/drho_0 (device array of nx * ny doubles, or NULL) and dJ/dgamma
 * (host, or NULL). */
int zg_adj_gradient(zg_adj *a, const zg_adj_params *prm, const double *rho, const double *u, const double *v,
                    const double *p, double *J, double *dJ_drho, double *dJ_dgamma);

/* Largest nx and ny that zg_rect_step_noalloc accepts. */
#define ZG_NOALLOC_MAX_AXIS 8192

/* One first-order step (accuracy 1, FP64, PARITY kernels) on the rectangle
 * of zg_mesh_rectangle, without a context and without allocating any memory.
 * It has no counterpart in the reference: it is for callers that cannot let
 * a library allocate device memory -- a program that hands out every byte of
 * each GPU from its own pool, or one that must not have an allocation
 * synchronise the device between its own stream operations.
 *
 * in[5] and out[5] are device arrays of nx * ny doubles each (density,
 * velocity x, velocity y, pressure, specific internal energy; cell (i, j)
 * at index i * ny + j, the order of the reference's base mesh,
 * amr_cells_gen.cpp:128-281); out must not overlap in.  The result equals
 * one zg_smf_update step of a context configured with the same parameters.
 * `dt` (device or pinned host memory, may be NULL) receives the step's dt.
 * The work is enqueued on `stream` (a cudaStream_t; NULL = default stream)
 * on CUDA device `device` and is asynchronous.
 *
 * Scratch: the CFL minimum, the dt and the coordinate tables live in one
 * fixed array of device memory inside the library (512 KiB on every
 * GPU that loads the library, held until the process exits).  nx and ny up
 * to ZG_NOALLOC_MAX_AXIS are accepted; larger meshes return
 * ZG_ERR_TOO_LARGE.  Every call resets the scratch it needs on `stream`
 * before use.  Every call looks up that array's address on the device (the
 * first lookup on a device may load the library's device code there; make
 * the first call before any stream capture on that device).  Calls that
 * overlap on one device -- on different streams, or from different host
 * threads -- share the one array and race: serialise them.  Every flux of
 * zg_flux is accepted.  A CUDA error already pending when the call starts
 * returns ZG_ERR_CUDA before anything is launched and is left pending. */
int zg_rect_step_noalloc(int device, int nx, int ny, double x_min, double x_max, double y_min,
                         double y_max, const int bounds[4], const zg_smf_params *p, const double *const in[5],
                         double *const out[5], double *dt, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* ZEPHYR_GPU_H */
