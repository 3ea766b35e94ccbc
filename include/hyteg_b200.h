/* C-ABI of the B200 matrix-free P1 geometric-multigrid hot path.
 *
 * Every entry point returns an int status (HG_OK = 0). Plain pointers and sizes only: no
 * C++ or PyTorch types cross this boundary. One hg_storage owns the macro-mesh topology,
 * all device memory of its functions and operators, and one CUDA stream; it is not
 * thread-safe, distinct storages are independent.
 *
 * Function data are kept on the device in the reference's per-primitive layout
 * (vertex / edge / face / cell arrays incl. ghost layers), see hg_primitive_layout.
 * The entry points replace these reference interfaces (paths within wagnandr/hyteg):
 *   hg_storage_create_cuboid   MeshInfo::meshCuboid + SetupPrimitiveStorage +
 *                              setMeshBoundaryFlagsOnBoundary(1,0,true)
 *                              (src/hyteg/mesh/MeshGenCuboid.cpp:32,
 *                               src/hyteg/primitivestorage/SetupPrimitiveStorage.cpp:37,735)
 *   hg_function_create         P1Function<real_t>(name, storage, minLevel, maxLevel)
 *                              (src/hyteg/p1functionspace/VertexDoFFunction.hpp:66-77)
 *   hg_communicate             VertexDoFFunction::communicate<S,R> in the six directions
 *                              (src/hyteg/p1functionspace/VertexDoFFunction.hpp:259-284)
 *   hg_interpolate_const       VertexDoFFunction::interpolate(constant, level, flag)
 *   hg_assign / hg_add         VertexDoFFunction::assign / add
 *                              (src/hyteg/p1functionspace/VertexDoFFunction.cpp:980,1077)
 *   hg_dot                     VertexDoFFunction::dotGlobal (VertexDoFFunction.cpp:1411)
 *   hg_operator_create         P1ConstantLaplaceOperator / P1ConstantMassOperator ctor
 *                              (src/hyteg/p1functionspace/P1ConstantOperator.hpp:165-166)
 *   hg_apply                   Operator::apply(src, dst, level, flag, updateType)
 *                              (src/hyteg/operators/Operator.hpp:73-80,
 *                               src/hyteg/p1functionspace/P1Operator.hpp:197-325)
 *   hg_residual                GeometricMultigridSolver residual: apply + assign{1,-1}
 *                              (src/hyteg/solvers/GeometricMultigridSolver.hpp:185-186)
 *   hg_smooth_sor              SORSmoothable::smooth_sor / smooth_sor_backwards
 *                              (src/hyteg/solvers/Smoothables.hpp:81-91), multicolour on the GPU
 *   hg_restrict                P1toP1LinearRestriction::restrict
 *                              (src/hyteg/gridtransferoperators/P1toP1LinearRestriction.cpp:163)
 *   hg_prolongate              P1toP1LinearProlongation::prolongate / prolongateAndAdd
 *                              (src/hyteg/gridtransferoperators/P1toP1LinearProlongation.cpp:189)
 *   hg_cg_solve                CGSolver::solve (src/hyteg/solvers/CGSolver.hpp:69-150)
 *   hg_gmg_*                   GeometricMultigridSolver (src/hyteg/solvers/GeometricMultigridSolver.hpp:36-259)
 */
#ifndef HYTEG_B200_H
#define HYTEG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  HG_OK = 0,
  HG_ERR_ARG = 1,      /* invalid argument (handle, level, flag, size) */
  HG_ERR_CUDA = 2,     /* CUDA runtime error or no device */
  HG_ERR_OOM = 3,      /* device allocation failed */
  HG_ERR_STATE = 4,    /* operation not valid in the current state */
  HG_ERR_NUMERIC = 5,  /* zero diagonal, breakdown */
  HG_ERR_INTERNAL = 6
};

/* DoFType bits (src/hyteg/types/types.hpp:35-44) */
#define HG_INNER 1u
#define HG_DIRICHLET 2u
#define HG_NEUMANN 4u
#define HG_FREESLIP 8u
#define HG_ALL 15u

/* primitive kinds */
#define HG_VERTEX 0
#define HG_EDGE 1
#define HG_FACE 2
#define HG_CELL 3

typedef struct hg_storage hg_storage;
typedef struct hg_mesh hg_mesh;

/* Text of the last error of the calling thread ("" if none). */
const char* hg_last_error(void);
/* Number of CUDA devices visible (0 on a machine without GPU); never fails. */
int hg_device_count(void);

int hg_storage_create_cuboid(const double lo[3], const double hi[3], int nx, int ny, int nz, int max_level,
                             hg_storage** out);
/* Explicit tetrahedral mesh: coords[3*nverts], tets[4*ncells] (vertex IDs in cell-frame order). */
int hg_storage_create_tets(int nverts, const double* coords, int ncells, const int* tets, int max_level,
                           hg_storage** out);
/* MeshInfo::meshCubedDomain (src/hyteg/mesh/MeshGenCubedDomain.cpp:115-383) + SetupPrimitiveStorage +
 * setMeshBoundaryFlagsOnBoundary(1, 0, true): unit cubes at the integer positions cubes[3*ncubes]
 * (duplicates ignored), split into 6 tetrahedra each (cube_type 0, the meshCuboid split) or 24
 * (cube_type 1: face-centre and cube-centre vertices). */
int hg_storage_create_cubed_domain(int ncubes, const int* cubes, int cube_type, int max_level, hg_storage** out);
/* MeshInfo::fromGmshFile (src/hyteg/mesh/MeshGenFromGmshFile.cpp:31-206) + SetupPrimitiveStorage: a
 * Gmsh 2.2 ASCII file (nodes; lines, triangles, tetrahedra and points). flags_from_file = 0 sets the
 * boundary flags from the geometry as setMeshBoundaryFlagsOnBoundary(1, 0, true) does; 1 keeps the
 * first tag of each line and triangle as the flag of that edge or face (others 0), as MeshInfo
 * does. A malformed file, a version other than 2.2, an unknown element type or a node outside every
 * tetrahedron fails with HG_ERR_ARG. */
int hg_storage_create_gmsh(const char* path, int max_level, int flags_from_file, hg_storage** out);
/* The storage's macro-mesh as a Gmsh 2.2 file (the wire format of a topology): vertices in ID order,
 * flagged edges and faces as lines and triangles, cells in frame order. Reading it back reproduces
 * the storage's primitives and their order; with flags_from_file = 0 the geometric boundary flags,
 * with 1 the written edge and face flags (vertices 0, as the reference's reader gives them). */
int hg_storage_write_gmsh(const hg_storage* s, const char* path);
int hg_storage_destroy(hg_storage* s);
/* counts[4] = {#vertices, #edges, #faces, #cells} */
int hg_storage_counts(const hg_storage* s, int counts[4]);
/* Use this CUDA stream (cudaStream_t) for all subsequent work; NULL = the storage's own stream. */
int hg_storage_set_stream(hg_storage* s, void* stream);
int hg_storage_synchronize(hg_storage* s);
/* Bytes of L2 that one group of macro-cells may occupy during the cell phase of an SOR sweep
 * (the four colour passes of a group run back to back); default: all macro-cells form one group. */
int hg_storage_set_l2_budget(hg_storage* s, int64_t bytes);
/* Number of device kernels this storage has launched so far. */
int hg_storage_launch_count(const hg_storage* s, unsigned long long* count);
/* Piecewise-constant diffusion coefficient per macro-cell (ncells values) for operators
 * created afterwards. */
int hg_storage_set_cell_coefficients(hg_storage* s, const double* k, int ncells);
/* Cell-phase schedule of the multicolour SOR: 0 (default) = one pass per sweep (z-wavefront over
 * the four colours, written to a second buffer of the level that then replaces the smoothed
 * function's buffer), 1 = four in-place colour passes, 2 = the single pass with shorter tiles
 * (32 x 12 instead of 32 x 24 / 28), 3 = four colour passes on copies of the cell arrays in the
 * colour-split order (each row ordered by x mod 4; the copies are made once per group of sweeps
 * of a multigrid smoothing step and the result is copied back). All give the same multicolour
 * sweep. */
int hg_storage_set_sor_schedule(hg_storage* s, int schedule);
/* Launch structure of the face, edge and vertex phases of the multicolour SOR (no counterpart in
 * the reference; the same sweep either way, bit for bit): on = 1 (default) runs each phase as one
 * launch, a block per primitive doing the phase's colours in turn, with the refresh of the face
 * boundary rows (before the faces) and of the vertex ghosts (before the vertices of a backward
 * sweep) folded in; on = 0 runs one launch per colour and per refresh. */
int hg_storage_set_sor_fused_phases(hg_storage* s, int on);
/* Whether hg_p2p1_stokes_minres[_mixed] runs the three velocity V-cycles of each preconditioner
 * application concurrently, one CUDA stream each, with one multigrid workspace per component, and
 * the Uzawa smoother (hg_p2p1_stokes_uzawa_*) its three components' velocity sweeps (no
 * counterpart in the reference, which applies them one after another; the iterates are the same
 * bit for bit): on = 1 (default) once the first application (or smoothing of a level) has run in
 * order, and for MINRES when the coarse level is solved directly on the device; on = 0 one after
 * another on the storage's stream. */
int hg_storage_set_concurrent_components(hg_storage* s, int on);
/* Autotuner (no counterpart in the reference): times the multicolour SOR under the four
 * schedules on every level in [min_level, max_level] (precision 8 or 4; `reps` timed groups of
 * three sweeps, the smoothing step of a V(3,3) cycle, after one warm-up group; CUDA events on the
 * storage's stream) and keeps the fastest schedule per level and precision, overriding
 * hg_storage_set_sor_schedule there. ms (nullable): 4 * (levels) times per sweep in ms, schedules
 * 0, 1, 2, 3 per level; chosen (nullable): the schedule kept per level. */
int hg_storage_autotune_sor(hg_storage* s, int min_level, int max_level, int precision, int reps, double* ms,
                            int* chosen);
/* The SOR schedule of one level and precision (8 or 4), as the autotuner sets it (-1: back to the
 * storage-wide hg_storage_set_sor_schedule). */
int hg_storage_set_sor_schedule_level(hg_storage* s, int level, int precision, int schedule);
/* Topology export: for kind HG_VERTEX ids[0..2]=unused, coords[3]; HG_EDGE ids[2]; HG_FACE ids[3];
 * HG_CELL ids[4]; flag = mesh boundary flag. */
int hg_primitive_vertices(const hg_storage* s, int kind, int prim, int ids[4], double coords[3], int* flag);
/* Neighbour list of a primitive: which = kind of neighbours (higher dimension), returns up to cap ids. */
int hg_primitive_neighbours(const hg_storage* s, int kind, int prim, int which, int* ids, int cap, int* count);
/* Offset and length of a primitive's array inside one function level buffer. */
int hg_primitive_layout(const hg_storage* s, int level, int kind, int prim, int64_t* offset, int64_t* size);
int hg_level_size(const hg_storage* s, int level, int64_t* n);

/* ---- Host-only view of the same discretization (no GPU needed): topology, per-level
 * layout, halo tables and stencil tables, for inspection and CPU-side verification. ---- */
int hg_mesh_create_cuboid(const double lo[3], const double hi[3], int nx, int ny, int nz, int max_level, hg_mesh** out);
int hg_mesh_create_tets(int nverts, const double* coords, int ncells, const int* tets, int max_level, hg_mesh** out);
/* The macro-mesh of the solve server's union hierarchies: `copies` disjoint copies of the unit
 * cube split into k^3 sub-cubes (meshCuboid), copy i translated by 2i along x; every kind of
 * primitive holds the copies' primitives copy after copy, each in a single cube's order. */
int hg_mesh_create_cuboid_copies(int k, int copies, int max_level, hg_mesh** out);
int hg_mesh_create_cubed_domain(int ncubes, const int* cubes, int cube_type, int max_level, hg_mesh** out);
int hg_mesh_create_gmsh(const char* path, int max_level, int flags_from_file, hg_mesh** out);
int hg_mesh_write_gmsh(const hg_mesh* m, const char* path);
int hg_mesh_destroy(hg_mesh* m);
int hg_mesh_counts(const hg_mesh* m, int counts[4]);
int hg_mesh_set_cell_coefficients(hg_mesh* m, const double* k, int ncells);
int hg_mesh_primitive_vertices(const hg_mesh* m, int kind, int prim, int ids[4], double coords[3], int* flag);
int hg_mesh_primitive_neighbours(const hg_mesh* m, int kind, int prim, int which, int* ids, int cap, int* count);
int hg_mesh_primitive_layout(const hg_mesh* m, int level, int kind, int prim, int64_t* offset, int64_t* size);
int hg_mesh_level_size(const hg_mesh* m, int level, int64_t* n);
/* Coordinates (3 per slot) of the micro-vertex each slot of a level buffer holds, and per slot
 * 1 = owned DoF, 0 = copy of a DoF owned elsewhere, -1 = alignment padding. */
int hg_mesh_slot_info(const hg_mesh* m, int level, double* xyz, signed char* owned, int64_t n);
/* The level-buffer slot of each entry of the packed owned-DoF order (hg_function_*_owned_async):
 * slots == null returns the count in *n; else *n must equal it. */
int hg_mesh_owned_slots(const hg_mesh* m, int level, int64_t* slots, int64_t* n);
/* Halo table of one group (0 vertex ghosts, 1 edge copies, 2 face boundary rows, 3 face ghost
 * layers, 4 cell closures): pass dst = src = NULL to query *n. */
int hg_mesh_halo_table(const hg_mesh* m, int level, int group, int64_t* dst, int64_t* src, int64_t* n);
/* Stencil of the owned points of one primitive (form 0 diffusion, 1 mass). Cells: 15 weights in
 * the order C E W N S NW SE TC TW TS TSE BC BE BN BNW. Faces: entries (layer, dx, dy, weight),
 * layer 0 = face, 1 + n = ghost layer of neighbour cell n. Edges / vertices: entries
 * (relative slot, weight). Entry 0 is the diagonal. cap = capacity of the output arrays. */
/* Verification of the colour-split SOR tables (schedule 3) on the host for level `level`: every
 * interior point of every colour is listed once, in order, and each of its 15 slots is the split
 * position of the right neighbour, recomputed from the neighbour's coordinates. points = interior
 * points checked; mismatches = points whose entry is wrong or missing, plus surplus entries. */
int hg_split_tables_check(int level, int64_t* points, int64_t* mismatches);
/* Verification of the device re-assembly's term lists (hg_operator_reassemble) on the host:
 * every stencil entry of (level, form) summed from its terms in order, compared bit for bit with
 * the assembled tables. targets / terms: sizes of the lists; mismatches: entries that differ. */
int hg_mesh_assembly_plan_check(const hg_mesh* m, int level, int form, int64_t* targets, int64_t* terms,
                                int64_t* mismatches);
int hg_mesh_cell_stencil(const hg_mesh* m, int level, int form, int cell, double w[15]);
int hg_mesh_face_stencil(const hg_mesh* m, int level, int form, int face, int* layer, int* dx, int* dy, double* w,
                         int cap, int* n);
int hg_mesh_low_stencil(const hg_mesh* m, int level, int form, int kind, int prim, int64_t* rel, double* w, int cap,
                        int* n);

/* precision: 8 = double, 4 = float */
int hg_function_create(hg_storage* s, int min_level, int max_level, int precision, int* fn);
int hg_function_destroy(hg_storage* s, int fn);
/* The address of a level buffer is stable except across multicolour SOR on that level under
 * schedule 0 (hg_storage_set_sor_schedule): the sweep writes the second buffer of the level and
 * the two are exchanged, so re-query the address after smoothing (an even number of sweeps
 * per level, as in a V(3,3) cycle, returns every buffer to its original address). */
int hg_function_device_ptr(hg_storage* s, int fn, int level, void** ptr);
/* Host <-> device copies of one level buffer (n elements of the function's precision). */
int hg_function_upload(hg_storage* s, int fn, int level, const void* host, int64_t n);
int hg_function_download(hg_storage* s, int fn, int level, void* host, int64_t n);
/* The upload enqueued on the caller's CUDA stream (a cudaStream_t), without waiting: the caller
 * orders it against the storage's stream with events and keeps the host buffer (pinned, for an
 * asynchronous copy) alive until it completes. For pipelining the next input's copy with the
 * current solve. */
int hg_function_upload_async(hg_storage* s, int fn, int level, const void* host, int64_t n, void* stream);
/* The download enqueued on the caller's CUDA stream, without waiting (the counterpart of
 * hg_function_upload_async): the caller orders it after the work that produced the values (an
 * event recorded on the storage's stream) and before the next work that changes them, and reads
 * the host buffer only after the copy completed. For pipelining a result's copy with the next
 * solve. */
int hg_function_download_async(hg_storage* s, int fn, int level, void* host, int64_t n, void* stream);
/* Packed transfers of the owned DoFs only (no counterpart in the reference, whose functions live
 * in host memory): every DoF of the level once, in level-buffer order (hg_mesh_owned_slots gives
 * the slot of each entry), n = hg_owned_count elements of the function's precision; about 9 %
 * fewer bytes than the level buffer on the 48-tet cube. The host copy runs on the caller's
 * stream, the packing on the storage's stream; a per-function staging buffer on the device
 * (allocated by the first call for a function and level; the level's table of owned runs by the
 * first hg_owned_count or transfer on that level) sits in between, and events order each
 * use of it after the previous one, so successive calls need no ordering by the caller beyond
 * that of the function itself. upload: the values are scattered into the owners' slots and every
 * copy slot is refreshed from its owner (the level buffer is then consistent), in order on the
 * storage's stream; the host buffer must stay alive (and pinned, for an asynchronous copy) until
 * the copy stream has passed the copy. download: the owners' values as of the storage's stream
 * at the call, in the host buffer once the caller's stream has passed the copy. */
int hg_owned_count(hg_storage* s, int level, int64_t* n);
int hg_function_upload_owned_async(hg_storage* s, int fn, int level, const void* host, int64_t n, void* stream);
int hg_function_download_owned_async(hg_storage* s, int fn, int level, void* host, int64_t n, void* stream);
int hg_communicate(hg_storage* s, int fn, int level);
int hg_interpolate_const(hg_storage* s, int fn, double value, int level, unsigned flag);
/* Built-in expressions at the flagged DoFs (then the halo is refreshed): expr 0 =
 * p0 sin(p1 pi x) sin(p1 pi y) sin(p1 pi z); expr 1 = p0 + p1 x + p2 y + p3 z. */
int hg_interpolate_expr(hg_storage* s, int fn, int level, unsigned flag, int expr, const double params[4]);
/* dst = sum_i scalars[i] * srcs[i]   (n <= 3) */
int hg_assign(hg_storage* s, int dst, int level, unsigned flag, int n, const double* scalars, const int* srcs);
/* dst += sum_i scalars[i] * srcs[i]  (n <= 3) */
int hg_add(hg_storage* s, int dst, int level, unsigned flag, int n, const double* scalars, const int* srcs);
/* dst = (precision of dst) src, or dst += src when add != 0; src and dst may differ in precision */
int hg_copy_cast(hg_storage* s, int dst, int src, int level, unsigned flag, int add);
int hg_dot(hg_storage* s, int a, int b, int level, unsigned flag, double* out);
/* hg_dot without any device allocation, for callers that may not allocate device memory while
 * they run (e.g. a service that commits its device-memory budget at start-up). No counterpart in
 * the reference. a, b: device pointers to one level buffer each (hg_function_device_ptr) of the
 * given precision (8 or 4); result: device pointer to one double, written on the storage's
 * stream (no synchronisation, no host copy). The scratch is a static device array of 65,536
 * partial sums: levels that need more blocks are rejected with HG_ERR_ARG. The call runs with the
 * storage's device current (the device that was current when the storage was created) and then
 * restores the caller's device. The first call on a storage looks up the array's device address
 * on that device, so make it before any stream capture. Every call shares the one array: calls
 * that overlap on the GPU (other streams, other threads) race. */
int hg_dot_noalloc(hg_storage* s, const void* a, const void* b, int precision, int level, unsigned flag,
                   double* result);

/* ---------------------------------------------------------------------------------------
 * P2 (quadratic Lagrange) operators. The P2 DoFs of level L (micro-vertices and micro-edge
 * midpoints of level L) are exactly the vertex DoFs of level L + 1, so a P2 function of levels
 * [a, b] is a function of levels [a + 1, b + 1] created with hg_function_create; its values at
 * even lattice coordinates are the vertex DoFs, the other seven parity classes the edge DoFs of
 * the reference's seven edge orientations (edgedofspace/EdgeDoFOrientation.hpp:29-39). The
 * reference stores the same values in separate vertex-DoF and edge-DoF arrays
 * (P2Function.hpp): a host adapter converts between the two layouts.
 * Replaces P2ConstantLaplaceOperator = P2ConstantOperator<P2FenicsForm<p2_diffusion,
 * p2_tet_diffusion>> (p2functionspace/P2ConstantOperator.hpp:154-157); form 0 only.
 * --------------------------------------------------------------------------------------- */
int hg_p2_operator_create(hg_storage* s, int form, int min_level, int max_level, int* op);
int hg_p2_operator_destroy(hg_storage* s, int op);
/* dst = A src at the flagged P2 DoFs of `level` (P2ConstantOperator.cpp:98-117, Replace). */
int hg_p2_apply(hg_storage* s, int op, int src, int dst, int level, unsigned flag);
/* r = b - A x at the flagged P2 DoFs of `level`. */
int hg_p2_residual(hg_storage* s, int op, int x, int b, int r, int level, unsigned flag);
/* One multicolour SOR sweep on P2 level `level` (P2ConstantOperator.cpp:1171-1235 smooth_sor).
 * Colours: the DoF's barycentric weights in ascending vertex-ID order (b0..b3) give the parity
 * class p = (b1&1) | (b2&1)<<1 | (b3&1)<<2; p = 0 is split into ((b1>>1) + 2(b2>>1) + 3(b3>>1))
 * mod 4, the edge DoFs form colours 3 + p. A pass updates one colour, every DoF of it from the
 * values at the start of the pass: x += omega (b - A x) / diag(A). backwards reverses the order. */
int hg_p2_smooth_sor(hg_storage* s, int op, int x, int b, double omega, int level, unsigned flag, int backwards);
/* Quadratic prolongation of fn from P2 level `level` to level + 1 (P2toP2QuadraticProlongation,
 * gridtransferoperators/P2toP2QuadraticProlongation.hpp), add != 0: prolongateAndAdd; and its
 * transpose, the restriction from P2 level `level` to level - 1 (P2toP2QuadraticRestriction). */
int hg_p2_prolongate(hg_storage* s, int fn, int level, unsigned flag, int add);
int hg_p2_restrict(hg_storage* s, int fn, int level, unsigned flag);
/* P2-P1 Taylor-Hood Stokes operator (P2P1TaylorHoodStokesOperator, composites/
 * P2P1TaylorHoodStokesOperator.hpp:33-84): the P2 Laplace per velocity component and the
 * divergence blocks P2ToP1ConstantDivOperator / P1ToP2ConstantDivTOperator (p2_to_p1_tet_div_tet,
 * p1_to_p2_tet_divt_tet). Velocity: three P2 functions; pressure: a P1 function whose level L is
 * the pressure of P2 level L. Destroy with hg_p2_operator_destroy.
 * apply: v_k = A u_k + D_k^T p at the velocity DoFs of flag_velocity, q = sum_k D_k u_k at the
 * pressure DoFs of flag_pressure.
 * minres: MinResSolver (solvers/MinresSolver.hpp:63-125) on level L with a block-diagonal
 * preconditioner (one symmetric P2 V(nu, nu) cycle per velocity component, inverse lumped P1
 * mass for the pressure) to the relative preconditioned residual tol; the Dirichlet values of u
 * are kept, the pressure is returned with zero mean. */
int hg_p2p1_stokes_create(hg_storage* s, int min_level, int max_level, int* op);
int hg_p2p1_stokes_apply(hg_storage* s, int op, const int u[3], int p, const int v[3], int q, int level,
                         unsigned flag_velocity, unsigned flag_pressure);
int hg_p2p1_stokes_minres(hg_storage* s, int op, const int u[3], int p, const int f[3], int g, int level, int nu,
                          int max_iter, double tol, int* iterations, double* rel_residual, double* history,
                          int history_cap);
/* The same with the preconditioner's V-cycles in FP32 (precondition_precision 4: FP32 storage and
 * arithmetic inside the cycles, coarse CG in FP64) while MINRES, the operator and the residual
 * stay FP64; precondition_precision 8 equals hg_p2p1_stokes_minres. */
int hg_p2p1_stokes_minres_mixed(hg_storage* s, int op, const int u[3], int p, const int f[3], int g, int level, int nu,
                                int max_iter, double tol, int precondition_precision, int* iterations,
                                double* rel_residual, double* history, int history_cap);
/* Geometric multigrid on the whole Taylor-Hood system (GeometricMultigridSolver with
 * P2P1TaylorHoodStokesOperator, GeometricMultigridSolver.hpp:136-235) with the Uzawa smoother
 * (UzawaSmoother.hpp:287-423, block-Laplace variant without stabilisation: r_u = f - D^T p;
 * velocity_sweeps forward P2 SOR sweeps per component; p += omega (g - D u) / diag(PSPG)) and the
 * composite transfers (P2P1StokesToP2P1StokesRestriction / Prolongation.hpp: quadratic on the
 * velocity, linear on the pressure). Velocity DoFs flagged Inner | Neumann are unknowns, every
 * pressure DoF is one (all-inner, P2P1TaylorHoodFunction.hpp:61). The coarsest level is solved by
 * the pseudo-inverse of the operator on its unknowns when it has at most 1024 of them, else by
 * hg_p2p1_stokes_minres (nu = 2) to a relative residual of 1e-11, where the reference uses an LU
 * solver; the operator must then cover level 0. u, f: velocity P2 functions,
 * p, g: pressure P1 functions, covering [min_level, max_level].
 *   smooth:   one UzawaSmoother::solve step on level
 *   solve:    one V(pre, post) cycle
 *   solve_to: cycles to the relative residual tol (over the unknowns) */
int hg_p2p1_stokes_uzawa_gmg_create(hg_storage* s, int op, int min_level, int max_level, int pre_smooth,
                                    int post_smooth, double omega, int velocity_sweeps, int* gmg);
int hg_p2p1_stokes_uzawa_gmg_destroy(hg_storage* s, int gmg);
int hg_p2p1_stokes_uzawa_smooth(hg_storage* s, int gmg, const int u[3], int p, const int f[3], int g, int level);
/* estimateUzawaRelaxationParameter (UzawaSmoother.hpp:52-68): the spectral radius of
 * M_lumped^-1 D S D^T (S: the smoother's velocity sweeps from zero) by power_iterations power
 * iterations (SpectrumEstimation.hpp:57-81) from seeded uniform [0, 1) values. */
int hg_p2p1_stokes_uzawa_estimate_omega(hg_storage* s, int gmg, int level, int power_iterations, uint64_t seed,
                                        double* omega);
int hg_p2p1_stokes_uzawa_gmg_solve(hg_storage* s, int gmg, const int u[3], int p, const int f[3], int g, int level);
int hg_p2p1_stokes_uzawa_gmg_solve_to(hg_storage* s, int gmg, const int u[3], int p, const int f[3], int g, int level,
                                      double tol, int max_iter, int* iterations, double* rel_residual, double* history,
                                      int history_cap);

/* P2 geometric multigrid (GeometricMultigridSolver with P2ConstantLaplaceOperator, the P2 SOR
 * above and the quadratic transfers; GeometricMultigridSolver.hpp:136-235), FP64. x, b: P2
 * functions covering [min_level, max_level]. solve: one cycle; solve_to: cycles to the relative
 * residual tol. The coarsest level is solved exactly when it has at most 1024 unknowns (the
 * inverse of the operator on them, built once), else by CG with coarse_max_iter / coarse_tol.
 * With the exact coarse solve, cycles are captured as CUDA graphs and replayed (default on;
 * the first cycle with a given set of buffers runs eagerly). set_graphs(0) turns that off. */
int hg_p2_gmg_create(hg_storage* s, int op, int min_level, int max_level, int pre_smooth, int post_smooth,
                     double omega, int coarse_max_iter, double coarse_tol, int* gmg);
int hg_p2_gmg_destroy(hg_storage* s, int gmg);
int hg_p2_gmg_solve(hg_storage* s, int gmg, int x, int b, int level);
int hg_p2_gmg_solve_to(hg_storage* s, int gmg, int x, int b, int level, double tol, int max_iter, int* iterations,
                       double* rel_residual, double* history, int history_cap);
int hg_p2_gmg_set_graphs(hg_storage* s, int gmg, int enable);

/* ---------------------------------------------------------------------------------------
 * Solve server (continuous batching). No counterpart in the reference, which solves one
 * problem per program run; this serves a stream of independent P1 Poisson solves.
 * A request is the unit cube split into k x k x k sub-cubes of 6 tetrahedra (meshCuboid),
 * refined to `level`, Dirichlet 0 on the boundary, constant coefficient, right-hand side
 * uniform[-1,1] at the inner DoFs from `seed` (hg_function_fill_random), x0 = 0, solved to the
 * relative residual `tol` with V(3,3) cycles (precision 8) or FP64 defect correction around
 * FP32 V(3,3) cycles (precision 4). `workers` threads scan the queue in arrival order and start
 * the first request that can start: on an idle resident hierarchy of its shape, or on a new one
 * built for it when its shape has none and its device footprint fits `hbm_budget_bytes`. A
 * request whose shape's hierarchies are all busy waits for one while the requests behind it may
 * pass it; a request waiting for memory is passed by none. Each running request has its own CUDA
 * stream, concurrent with the others.
 * --------------------------------------------------------------------------------------- */
typedef struct hg_server hg_server;
int hg_server_create(int workers, int64_t hbm_budget_bytes, int precision, hg_server** out);
int hg_server_destroy(hg_server* srv);
/* Build one resident hierarchy of shape (k, level) ahead of the first request (its cycle's CUDA
 * graph is captured here, so that requests only replay it). */
int hg_server_prewarm(hg_server* srv, int k, int level);
int hg_server_submit(hg_server* srv, int k, int level, double coefficient, uint64_t seed, double tol, int max_iter,
                     int keep_solution, int64_t* id);
/* Block until the request has finished (timeout < 0: no limit); *done = 1 when it has. */
int hg_server_wait(hg_server* srv, int64_t id, double timeout_seconds, int* done);
/* status: 0 queued, 1 running, 2 done, -1 failed (message in hg_last_error after this call
 * returns HG_ERR_STATE); times: submit, admission, start of the iteration (after the stencils
 * and the right-hand side are set up), end, in seconds since hg_server_create. */
int hg_server_result(hg_server* srv, int64_t id, int* status, int* iterations, double* rel_residual, double times[4],
                     int64_t* inner_dofs);
/* Batched solves (no counterpart in the reference): requests of levels up to max_level (-1, the
 * default: none) that find no single hierarchy of their shape idle are solved together when a
 * union hierarchy of their shape is idle and at least two requests of that shape are queued; the
 * smallest idle union that takes them all is used, else the largest. A union hierarchy
 * (hg_server_prewarm_batch) is one storage holding `copies` disjoint copies of the shape's
 * macro-mesh: up to `copies` queued requests of the shape share one solve, every kernel launch of
 * which covers all of them. Copy i takes request i's coefficient and right-hand side, its
 * residual norms are its own, and the coarse-grid CG runs one block per copy; each request stops
 * at its own tolerance (its solution is taken at that iteration), so it gets the iterations,
 * residual and solution it gets alone, bit for bit.
 * hg_server_request_batch: the number of requests solved together with request id (itself
 * included; 1 when it was solved alone). */
int hg_server_set_batching(hg_server* srv, int max_level);
int hg_server_prewarm_batch(hg_server* srv, int k, int level, int copies);
int hg_server_request_batch(hg_server* srv, int64_t id, int* batch_size);
/* Whether request id's hierarchy was built when it was admitted (1: its shape had no resident
 * hierarchy, so its setup time includes building one: storage, tables, stencils and the first
 * cycles) or was a resident one (0: its setup is the re-assembly of the stencils for its
 * coefficient). */
int hg_server_request_setup(hg_server* srv, int64_t id, int* built_hierarchy);
/* Level buffer of the solution (requests submitted with keep_solution); *size = elements. */
int hg_server_solution(hg_server* srv, int64_t id, double* host, int64_t n, int64_t* size);
/* admitted, completed, failed, resident idle hierarchies, their bytes, peak bytes in use. */
int hg_server_stats(hg_server* srv, int64_t stats[6]);
/* Seeded uniform [lo, hi) values at the DoFs of the flagged primitives, then a halo refresh; the
 * values depend only on (seed, slot), so equal topologies give equal vectors. */
int hg_function_fill_random(hg_storage* s, int fn, int level, unsigned flag, uint64_t seed, double lo, double hi);

/* form: 0 = diffusion (Laplace, scaled by the per-cell coefficient), 1 = mass, 2 = PSPG
 * stabilisation -tau grad p . grad q with tau = |T|^(2/3) / 12 per micro-cell (P1PSPGOperator,
 * p1functionspace/P1ConstantOperator.hpp:201-208; forms/form_fenics_generated/p1_tet_pspg_tet.h) */
int hg_operator_create(hg_storage* s, int form, int min_level, int max_level, int* op);
int hg_operator_destroy(hg_storage* s, int op);
/* Re-assembles the operator's stencils on all its levels from the storage's current cell
 * coefficients (hg_storage_set_cell_coefficients). on_device = 0: on the host, then uploaded (as
 * at creation). on_device = 1: from per-entry lists of element-matrix terms, one kernel per level
 * on the storage's stream. The first call builds the lists (host work similar to one host
 * assembly). The results are bit-identical to the host assembly. Only the diffusion form
 * depends on the coefficients; the other forms are left as they are. */
int hg_operator_reassemble(hg_storage* s, int op, int on_device);
/* update: 0 = Replace, 1 = Add */
int hg_apply(hg_storage* s, int op, int src, int dst, int level, unsigned flag, int update);
/* The per-primitive-kind kernels of hg_apply without (refresh = 0) or with (1) the preceding
 * halo refresh: kinds is a bit set (1 << HG_VERTEX | 1 << HG_EDGE | 1 << HG_FACE | 1 << HG_CELL).
 * Replaces the per-macro-primitive kernel calls of P1ConstantOperator
 * (apply_cell_generated / apply_face3D_generated, P1ConstantOperator.cpp:202-336). */
int hg_apply_primitives(hg_storage* s, int op, int src, int dst, int level, unsigned flag, int update, int kinds,
                        int refresh);
/* r = b - A x on the flagged primitives */
int hg_residual(hg_storage* s, int op, int x, int b, int r, int level, unsigned flag);
int hg_smooth_sor(hg_storage* s, int op, int dst, int rhs, double omega, int level, unsigned flag, int backwards);
/* The phases of one SOR sweep restricted to the selected primitive kinds (bit set as in
 * hg_apply_primitives), with (refresh = 1) or without the halo refreshes. */
int hg_smooth_sor_primitives(hg_storage* s, int op, int dst, int rhs, double omega, int level, unsigned flag,
                             int backwards, int kinds, int refresh);
/* fn(src_level - 1) = R fn(src_level) */
int hg_restrict(hg_storage* s, int fn, int src_level, unsigned flag);
/* fn(src_level + 1) = P fn(src_level)   (add != 0: +=) */
int hg_prolongate(hg_storage* s, int fn, int src_level, unsigned flag, int add);

/* Conjugate gradients on one level (flag Inner|Neumann|Freeslip as in the reference).
 * Stops when sqrt(r.r) < tol or after max_iter iterations. */
int hg_cg_solve(hg_storage* s, int op, int x, int b, int level, int max_iter, double tol, int* iterations,
                double* final_residual);

/* Geometric multigrid V/W-cycles: SOR smoother (multicolour, omega), CG coarse solver. */
int hg_gmg_create(hg_storage* s, int op, int min_level, int max_level, int pre_smooth, int post_smooth,
                  double omega, int cycle_type /*0 V, 1 W*/, int coarse_max_iter, double coarse_tol,
                  int precision, int* gmg);
int hg_gmg_destroy(hg_storage* s, int gmg);
/* One cycle: x <- MG(x, b) on max_level (x, b of the solver's precision). */
int hg_gmg_solve(hg_storage* s, int gmg, int x, int b, int level);
/* Device-timed phases of the multigrid (walberla::WcTimingTree around GeometricMultigridSolver,
 * GeometricMultigridSolver.hpp:127-234, and CGSolver): on = 1 starts an empty tree (cycles then run
 * eagerly, not from graphs), 0 drops it. Nodes as in the reference: "Geometric Multigrid Solver" >
 * "Level L" > "Smoother" (count = sweeps), "Restriction", "Prolongation", "Coarse Grid Solver" >
 * "CG Solver"; intervals are CUDA events on the storage's stream. */
int hg_gmg_set_timing(hg_storage* s, int gmg, int on);
/* The tree as JSON (waLBerla TimingTree layout with "Remainder" nodes, seconds): waits for the
 * recorded events; *len = the full length; buf (nullable) receives up to cap-1 bytes and a 0. */
int hg_gmg_timing_json(hg_storage* s, int gmg, char* buf, int64_t cap, int64_t* len);
/* Cycles are captured as CUDA graphs and replayed (default on) when the coarse solve runs on the
 * device (a coarse level with only vertex and edge DoFs, whose CG runs in one block, or a
 * compact coarse cycle that covers it) and pre + post smoothing steps are even. The first cycle with a given set of buffers runs eagerly, the second is
 * captured; any change of a buffer address (for example an odd number of SOR sweeps on one of
 * the functions elsewhere) selects or captures another graph. Results are identical either way. */
int hg_gmg_set_graphs(hg_storage* s, int gmg, int enable);
/* Compact coarse cycle of a V-cycle solver: the levels from the coarsest up to the highest one
 * with at most max_dofs unknowns per group (the whole mesh, or each copy of a storage of
 * disjoint copies after hg_gmg_set_coarse_groups) run as ONE launch per cycle: smoothing,
 * residuals, transfers and the coarse CG of those levels on owner-indexed vectors in device
 * scratch, one block (cluster_blocks 1) or one thread-block cluster of 2, 4 or 8 blocks per
 * group. Same multicolour order and coarse CG as the level-by-level cycle, so the iterates agree
 * up to rounding (the sums run in another order). max_dofs 0 turns it off; the default is 6000
 * unknowns and one block. Not used while the timing tree is on, nor for W-cycles.
 * Replaces the levels' share of GeometricMultigridSolver::solveRecursively
 * (src/hyteg/solvers/GeometricMultigridSolver.hpp:136-235) in one launch. */
int hg_gmg_set_compact(hg_storage* s, int gmg, int max_dofs, int cluster_blocks);
/* The highest level the compact coarse cycle covers, -1 when none. */
int hg_gmg_compact_top(hg_storage* s, int gmg, int* top);
/* Iterate to ||b - A x|| <= tol ||b - A x0|| (at most max_iter iterations); x, b are FP64. An FP64
 * solver repeats its cycle; an FP32 solver (precision 4) runs FP64 defect correction: r = b - A x
 * in FP64, one FP32 cycle on A e = r from e = 0 (its coarse CG in FP64), x += e in FP64.
 * history (nullable) receives the relative residual after each iteration. */
int hg_gmg_solve_to(hg_storage* s, int gmg, int x, int b, int level, double tol, int max_iter, int* iterations,
                    double* rel_residual, double* history, int history_cap);

#ifdef __cplusplus
}
#endif

#endif /* HYTEG_B200_H */
