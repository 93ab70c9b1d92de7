/*
 * salvus_b200.h -- C ABI of the B200 spectral-element time step.
 *
 * The reference boundary is Salvus's C++ plugin API: the time loop in
 * src/cxx/Main.cpp:45-66 calls, once per step,
 *   Problem::assembleIntoGlobalDof   (include/Problem/Problem.h:84-90,
 *                                     src/cxx/Problem/Problem.cpp:143-214)
 *   Problem::applyInverseMassMatrix  (Problem.h:112, Order2Newmark.cpp:68-83)
 *   Problem::takeTimeStep            (Problem.h:120-121, Order2Newmark.cpp:85-114)
 * on elements built by Element::Factory (src/cxx/Element/Element.cpp:117-304)
 * from a DMPlex mesh (src/cxx/Mesh/Mesh.cpp:53-86,361-452) and an Exodus
 * model (src/cxx/Model/ExodusModel.cpp:422-471).  This ABI replaces those
 * calls; every entry point below names the reference interface it replaces.
 *
 * Conventions: plain C types only.  Every function returns SALVUS_OK (0) or a
 * negative status and records a message readable with salvus_last_error()
 * (thread-local).  The library owns device memory; callers own host arrays.
 * Handles are opaque.  Calls on one problem are serialised on that problem's
 * CUDA stream.
 */
#ifndef SALVUS_B200_H
#define SALVUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SALVUS_OK 0
#define SALVUS_E_INVALID (-1)     /* bad argument / mesh (reference: std::runtime_error) */
#define SALVUS_E_OOM (-2)         /* device or host allocation failed */
#define SALVUS_E_CUDA (-3)        /* CUDA runtime error */
#define SALVUS_E_TIMEOUT (-4)     /* a bounded device wait gave up */
#define SALVUS_E_NONFINITE (-5)   /* NaN / Inf detected in a wavefield */
#define SALVUS_E_STATE (-6)       /* call out of order (e.g. no dt set) */
#define SALVUS_E_UNSUPPORTED (-7) /* order / shape / physics not built */
#define SALVUS_E_NOT_FOUND (-8)   /* source / receiver outside the mesh */

enum salvus_shape { SALVUS_QUAD = 0, SALVUS_HEX = 1, SALVUS_TRI = 2, SALVUS_TET = 3 };
enum salvus_physics { SALVUS_ACOUSTIC = 0, SALVUS_ELASTIC3D = 1, SALVUS_ELASTIC2D = 2,
                      SALVUS_COUPLED2D = 3 };
enum salvus_precision { SALVUS_FP32 = 0, SALVUS_FP64 = 1 };
enum salvus_field { SALVUS_FIELD_U = 0, SALVUS_FIELD_V = 1, SALVUS_FIELD_A = 2,
                    SALVUS_FIELD_A_PREV = 3 };
enum salvus_source_kind { SALVUS_SOURCE_FORCE = 0, SALVUS_SOURCE_MOMENT_TENSOR = 1 };
enum salvus_run_mode { SALVUS_RUN_PLAIN = 0, SALVUS_RUN_GRAPH = 1 };

/* Mesh description.  Replaces Mesh::read + ExodusModel::read +
 * Mesh::setupGlobalDof (Mesh.cpp:53-86, 361-452; ExodusModel.cpp:37,422).
 * cells use the reference's right-hand (PETSc) vertex order:
 *   quad v0(-,-) v1(+,-) v2(+,+) v3(-,+)                  (QuadP1.h:98-108)
 *   hex  v0(-,-,-) v1(-,+,-) v2(+,+,-) v3(+,-,-)
 *        v4(-,-,+) v5(+,-,+) v6(+,+,+) v7(-,+,+)         (HexP1.cpp:86-122)
 *   tri  v0 -> (-1,-1), v1 -> (1,-1), v2 -> (-1,1), counter-clockwise
 *                                                          (TriP1.cpp:56-94)
 *   tet  v0 -> (0,0,0), v1 -> (0,1,0), v2 -> (1,0,0), v3 -> (0,0,1) with
 *        det[v2-v0; v1-v0; v3-v0] > 0                     (TetP1.cpp:91-150)
 * Simplices are the P3 mass-lumped elements (12-node triangle, 50-node
 * tetrahedron; order must be 3); elastic3d runs on hexahedra and tetrahedra,
 * elastic2d on quadrilaterals.
 * params are per element, per element vertex (Exodus NAME_0..NAME_k):
 *   acoustic : [1][n_elements][nv]  VP                    (Scalar.cpp:23-25)
 *   elastic3d: [3][n_elements][nv]  RHO, VP, VS  (isotropic form of
 *              Elastic3D.cpp:33-54 with VPV=VPH=VP, VSV=VSH=VS, ETA=1), or
 *              with flag SALVUS_MESH_ELASTIC_TI the reference's six
 *              [6][n_elements][nv] RHO, VPV, VPH, VSV, VSH, ETA: transversely
 *              isotropic with a vertical axis, c11 = c22 = rho VPH^2,
 *              c33 = rho VPV^2, c44 = c55 = rho VSV^2, c66 = rho VSH^2,
 *              c12 = c11 - 2 c66, c13 = c23 = ETA (c11 - 2 c44)
 *              (Elastic3D.cpp:42-53, stress :106-118)
 *   elastic2d: [5][n_elements][4]   RHO, C11, C13, C33, C55
 *              (Elastic2D.cpp:29-37; fields ux, uy)
 *   coupled2d: [7][n_elements][4]   FLUID, VP, RHO, C11, C13, C33, C55:
 *              quadrilaterals of both kinds in one mesh, FLUID = 1 (same at
 *              all four vertices) marks a fluid element (Scalar physics on
 *              VP; RHO feeds the coupling), 0 a solid one (Elastic2D); fields
 *              per node [u, ux, uy].  Neighbours of the other kind couple
 *              through the ElasticToAcoustic2D / AcousticToElastic2D surface
 *              integrals (ElasticToAcoustic.cpp:17-41,
 *              AcousticToElastic2D.cpp:18-60) and share the reference's
 *              single summed mass (Order2Newmark.cpp:38-52). */
/* salvus_mesh_desc.flags: build only the FP32 stiffness records (halves the
 * per-mesh geometry memory; FP64 problems and the FP64 eigenvalue estimate
 * are then unavailable on that mesh). */
#define SALVUS_MESH_FP32_ONLY 1
/* salvus_mesh_desc.flags: elastic3d params are the six transversely isotropic
 * parameters (see above).  A model that is isotropic everywhere (VPH = VPV,
 * VSH = VSV, ETA = 1) runs the isotropic kernels; others store five folded
 * constants per point.  Tetrahedra with such material run on CUDA cores;
 * problem groups take isotropic meshes only. */
#define SALVUS_MESH_ELASTIC_TI 2
/* salvus_mesh_desc.flags: keep per-point inverse Jacobians for elastic
 * hexahedra even when every element is a parallelepiped.  By default such
 * meshes store one inverse Jacobian per element and FP32 records of the
 * material alone (12 instead of 48 bytes per point with the connectivity);
 * with SALVUS_HEX_STEP=fused in the environment the FP32 step also advances
 * each element's interior nodes inside the stiffness kernel (bitwise the
 * same result; measured slower on the order-4 benchmark mesh). */
#define SALVUS_MESH_PER_POINT_GEOMETRY 4

typedef struct {
  int32_t shape;   /* enum salvus_shape */
  int32_t order;   /* polynomial order: quad 1..10, hex 1..6, tri / tet 3 */
  int32_t physics; /* enum salvus_physics */
  int32_t reserved; /* flags: SALVUS_MESH_FP32_ONLY | SALVUS_MESH_ELASTIC_TI |
                       SALVUS_MESH_PER_POINT_GEOMETRY */
  int64_t n_vertices;
  const double *vertices; /* [n_vertices][dim] */
  int64_t n_elements;
  const int64_t *cells;   /* [n_elements][nv]: quad 4, hex 8, tri 3, tet 4 */
  const double *params;
} salvus_mesh_desc;

/* One Ricker point source (Ricker::fire, Ricker.cpp:27-33; Source.h:75).
 * FORCE: comp[0..c-1] is the direction (c = 1 acoustic, 2 elastic 2-D,
 * 3 elastic 3-D; coupled2d: [fluid, x, y], of which the owning element's
 * components act).
 * MOMENT_TENSOR (elastic only, no reference counterpart): comp = [Mxx, Myy,
 * Mzz, Myz, Mxz, Mxy] in 3-D, [Mxx, Myy, Mxy] in 2-D (solid elements of
 * coupled2d meshes only); nodal force
 * f_{i,a} = sum_b M_ab dphi_i/dx_b (x_s). */
typedef struct {
  double location[3];
  double center_freq;
  double time_delay;
  double amplitude;
  int32_t kind;
  int32_t shot; /* which shot of a batched problem (0 for single-shot) */
  double comp[6];
} salvus_source;

typedef struct salvus_mesh salvus_mesh;
typedef struct salvus_problem salvus_problem;

const char *salvus_last_error(void);
/* Library build string (compile arch, version). */
const char *salvus_version(void);

/* ---- reference elements ---- */
/* Nodes, weights and derivative tables of one reference element:
 * *n_points = P; points [P][dim] reference coordinates; weights [P];
 * dphi [dim][P][P] with dphi[(k*P + i)*P + q] = d phi_i / d xi_k at point q.
 * Replaces TensorQuad::GllPointsForOrder / GllIntegrationWeightsForOrder /
 * setupGradientOperator (TensorQuad.cpp:51-142), the Hexahedra equivalents
 * (Hexahedra.cpp:75-130, 535-577), Triangle::QuadraturePoints /
 * QuadratureIntegrationWeight / setupGradientOperator (Triangle.cpp:24-54,
 * 244-254) and Tetrahedra::QuadraturePoints / QuadratureIntegrationWeights /
 * setupGradientOperator (Tetrahedra.cpp:66-99, 434-448).  Output pointers may
 * be NULL.  Needs no GPU. */
int salvus_element_tables(int32_t shape, int32_t order, int32_t *n_points, double *points,
                          double *weights, double *dphi);

/* ---- mesh ---- */
/* Flattens the mesh once: GLL connectivity by topological keys, FP64
 * Jacobians / material / diagonal mass computed on the GPU and stored in the
 * problem precision.  Replaces Problem::initializeElements (Problem.cpp:34-140),
 * Mesh::setupGlobalDof and Order2Newmark::initializeGlobalDofs
 * (Order2Newmark.cpp:32-66).  device < 0 builds the host-side numbering and
 * node coordinates only (no GPU needed); such a mesh cannot hold problems. */
int salvus_mesh_create(const salvus_mesh_desc *desc, int device, salvus_mesh **out);
int salvus_mesh_destroy(salvus_mesh *mesh);
/* Unique global GLL nodes G and components c. */
int salvus_mesh_info(const salvus_mesh *mesh, int64_t *n_nodes, int32_t *n_components,
                     int32_t *points_per_element);
/* Storage chosen for the mesh (no reference counterpart): *per_element_jacobian
 * = 1 when every element is a parallelepiped and one inverse Jacobian per
 * element is kept (elastic hexahedra, SALVUS_MESH_PER_POINT_GEOMETRY unset);
 * *gathered_nodes = the nodes the fused FP32 step assembles by node gather
 * when it advances the interior nodes in the stiffness kernel (fused
 * hexahedron step, fused shot-batched step), all G otherwise.
 * Either pointer may be NULL. */
int salvus_mesh_layout(const salvus_mesh *mesh, int32_t *per_element_jacobian,
                       int64_t *gathered_nodes);
/* Node coordinates [G][dim] (QuadP1::buildNodalPoints QuadP1.cpp:176-216,
 * HexP1::buildNodalPoints HexP1.cpp:312-354). */
int salvus_mesh_node_coords(const salvus_mesh *mesh, double *xyz);
/* Element-local to global node map [E][P] (the closure, Problem.cpp:302-318). */
int salvus_mesh_connectivity(const salvus_mesh *mesh, int64_t *conn);
/* Owning element (first in element order whose hull holds the point) and
 * reference coordinates of a physical point: QuadP1::checkHull +
 * inverseCoordinateTransform (QuadP1.cpp:8-92), HexP1 (HexP1.cpp:8-187), as
 * used by attachSource / attachReceiver.  Works on host-only meshes. */
int salvus_mesh_locate_point(const salvus_mesh *mesh, const double *xyz, int64_t *element,
                             double *ref);
/* Nodes on the outer boundary of the mesh (on element faces -- edges in
 * 2-D -- that belong to one element), ascending global ids; nodes may be NULL
 * to query the count: the point set Mesh::setupTopology collects from the
 * side sets and their closures (Mesh.cpp:286-312) when every side of the
 * mesh is in a side set. */
int salvus_mesh_boundary_nodes(const salvus_mesh *mesh, int64_t *count, int64_t *nodes);
/* Diagonal inverse mass [G] in FP64 (VecReciprocal, Order2Newmark.cpp:52). */
int salvus_mesh_inverse_mass(const salvus_mesh *mesh, double *mi);
/* Estimate lambda_max(M^-1 K) by power iteration on the GPU (FP64);
 * dt_crit = 2 / sqrt(lambda_max).  The reference has no quad/hex CFL
 * (Mesh.h:60 is the constant 1.0). */
int salvus_mesh_max_eigenvalue(salvus_mesh *mesh, int32_t iterations, uint64_t seed,
                               double *lambda_max);

/* ---- problem (one wavefield set on a mesh) ---- */
/* Replaces Problem::Factory + Order2Newmark (Problem.cpp:11,
 * Order2Newmark.cpp:116-118).  n_shots > 1 selects the shot-batched layout. */
int salvus_problem_create(salvus_mesh *mesh, int32_t precision, int32_t n_shots,
                          salvus_problem **out);
int salvus_problem_destroy(salvus_problem *p);
int salvus_problem_set_dt(salvus_problem *p, double dt);
/* Element::attachSource / Source::Factory (TensorQuad.cpp:270-284,
 * Hexahedra.cpp:448-464): first element in element order whose hull holds
 * the point, then the Newton inverse map. */
int salvus_problem_add_source(salvus_problem *p, const salvus_source *src);
/* Element::attachReceiver (TensorQuad.cpp:253-268, Hexahedra.cpp:429-446).
 * Receivers are shared by all shots.  Returns SALVUS_OK; samples of u are
 * taken after every step (FP64 sum of Lagrange-weighted nodes). */
int salvus_problem_add_receiver(salvus_problem *p, const double *xyz);
/* Capacity of the on-device seismogram ring, in steps (default 4096). */
/* Homogeneous Dirichlet boundary (HomogeneousDirichlet.cpp:14-79): every
 * element point on one of the listed global nodes has its stiffness row
 * zeroed (the source term still acts there), as the reference's
 * HomogeneousDirichlet mixin does for the DOFs on boundary vertices, edges and
 * faces of its elements.  n = 0 clears.  Not for shot-batched problems. */
int salvus_problem_set_dirichlet(salvus_problem *p, int64_t n, const int64_t *nodes);
int salvus_problem_set_seismogram_capacity(salvus_problem *p, int64_t steps);
/* Host <-> device field copies, [G][c] FP64 for one shot
 * (Problem::insertElementalFieldIntoMesh Problem.cpp:286-300,
 * getFieldOnElement Problem.cpp:302-318). */
int salvus_problem_set_field(salvus_problem *p, int32_t field, int32_t shot, const double *vals);
int salvus_problem_get_field(salvus_problem *p, int32_t field, int32_t shot, double *vals);

/* ---- the reference's three per-step calls (literal form) ---- */
/* a = f(t_n) - K u, assembled; t_n = step * dt.
 * Problem::assembleIntoGlobalDof (Problem.cpp:143-214). */
int salvus_assemble(salvus_problem *p);
/* a <- M^-1 a.  Order2Newmark::applyInverseMassMatrix (Order2Newmark.cpp:68-83). */
int salvus_apply_inverse_mass(salvus_problem *p);
/* v += dt/2 (a + a_prev); u += dt v + dt^2/2 a; a_prev = a; step += 1;
 * receivers sampled.  Order2Newmark::takeTimeStep (Order2Newmark.cpp:85-114). */
int salvus_take_time_step(salvus_problem *p);

/* ---- fused forms ---- */
/* One fused step (the three calls above in one stiffness + one gather/update
 * launch).  Same result as the three-call sequence. */
int salvus_step(salvus_problem *p);
/* n steps of the Main.cpp:45-66 loop; mode PLAIN launches each step from the
 * host, GRAPH replays captured CUDA graphs of steps: a 32-step graph n / 32
 * times, then a graph of the remaining steps when there are at least 8
 * (the last remainder length is kept), else host launches for them.  In
 * the graphs each step's receivers run on a second stream of the problem,
 * overlapped with the next step's stiffness launch, and every graph ends
 * with them joined to the problem's stream (results are those of single
 * salvus_step calls). */
int salvus_run(salvus_problem *p, int64_t n_steps, int32_t mode);
/* Capture (without running) the graphs a GRAPH run of n_steps replays, so
 * that the run itself launches no capture.  No reference counterpart. */
int salvus_problem_prepare_run(salvus_problem *p, int64_t n_steps);
int salvus_synchronize(salvus_problem *p);
int64_t salvus_problem_step_index(const salvus_problem *p);
/* Shot batching (n_shots > 1; FP32 acoustic quads): picks, by timing on this
 * problem, the shot lanes and elements per CTA of the batched stiffness
 * kernel and the shot lanes and nodes per CTA of the batched gather/update
 * (no reference counterpart; the reference runs one source set per run).
 * Runs automatically before the first batched step; results are cached per
 * (order, shots, elements, device).  Single-shot problems report fixed
 * values.  SALVUS_BATCH_CONFIG="i,j" pins the choice. */
int salvus_problem_autotune(salvus_problem *p, int32_t *stiff_shot_lanes,
                            int32_t *stiff_elements, int32_t *gather_shot_lanes,
                            int32_t *gather_nodes);
/* Step form the problem runs, as chosen by the autotuners (no reference
 * counterpart; the reference has one form of Problem::takeTimeStep):
 *   form  SALVUS_STEP_PLAIN (stiffness kernel, then the node gather / Newmark
 *         update over every node) or SALVUS_STEP_FUSED_INTERIOR (the
 *         stiffness kernel also advances each element's interior nodes; the
 *         gather covers the shared nodes only).  Both forms give bitwise the
 *         same fields.
 *   elements_per_cta  elements per CTA of the stiffness kernel where it is
 *         tuned (FP32 parallelepiped elastic hexahedra: 128 / (N+1)^2 or twice
 *         that; shot-batched quads: the batched kernel's elements), else 0.
 * FP32 single-shot elastic hexahedron meshes of parallelepipeds are tuned by
 * timing every admissible (form, CTA width) on scratch copies of the fields
 * before the first run (cached per mesh size and device for the process;
 * SALVUS_HEX_CONFIG="form,wide" pins the choice, SALVUS_HEX_STEP=fused or
 * plain forces the form).  Runs the tuning if it has not run yet. */
#define SALVUS_STEP_PLAIN 0
#define SALVUS_STEP_FUSED_INTERIOR 1
int salvus_problem_step_config(salvus_problem *p, int32_t *form, int32_t *elements_per_cta);
/* Device status of the problem (synchronises its stream): SALVUS_OK,
 * SALVUS_E_NONFINITE when the displacement field held a NaN / Inf at one of
 * the finite checks (after every 32 steps of salvus_run / salvus_step /
 * salvus_take_time_step: an unstable time step or a non-finite input field),
 * or SALVUS_E_TIMEOUT when a bounded device wait gave up.  The same status is
 * returned by salvus_synchronize, salvus_problem_get_field and
 * salvus_get_seismograms.  clear != 0 resets the status word afterwards (the
 * fields are left as they are: set them again before continuing).  The
 * reference reports such failures as exceptions caught in main
 * (Main.cpp:70-74). */
int salvus_problem_status(salvus_problem *p, int32_t clear);
/* Bound, in SM clock cycles, of every device-side wait in this problem's
 * kernels (the tensor-core simplex kernels' hand-offs between their MMA
 * issuer and worker warps); <= 0 restores the default 2^31 (about a
 * second).  A wait that runs out records its code in the status word
 * (SALVUS_E_TIMEOUT, results invalid) and the kernel returns cleanly after
 * draining its own MMAs under the default bound.  A short limit makes waits
 * give up on purpose: for testing the timeout path. */
int salvus_problem_set_wait_limit(salvus_problem *p, int64_t cycles);
/* Testing the timeout path (no reference counterpart): with enable != 0 the
 * worker warps of the tensor-core simplex kernels first wait on a barrier
 * that nothing arrives on, so every such launch runs out of its wait limit,
 * returns cleanly and the problem reports SALVUS_E_TIMEOUT (results
 * invalid); enable = 0 restores normal launches.  Other kernels ignore it. */
int salvus_problem_hold_device_waits(salvus_problem *p, int32_t enable);
/* The problem's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events after this problem's kernels. */
int salvus_problem_stream(const salvus_problem *p, void **stream);

/* Seismograms [n_shots][n_receivers][c][n_steps] FP64 for steps
 * [first_step, first_step + n_steps) still held in the ring. */
int salvus_get_seismograms(salvus_problem *p, int64_t first_step, int64_t n_steps, double *out);
int salvus_problem_info(const salvus_problem *p, int32_t *n_shots, int32_t *n_receivers,
                        int32_t *n_components);

/* ---- allocation-free stiffness action ---- */
/* a = -K u, assembled over the mesh (no mass, no sources), for callers that
 * cannot allocate device memory while they run: frameworks that own all
 * device memory through their own pool, or code that must not touch the
 * allocator mid-run.  This entry point has no counterpart in the reference.
 * u and a are the caller's device buffers, [G][c] in `precision` (FP32 or
 * FP64); stream is a cudaStream_t or NULL.  The call is asynchronous on that
 * stream and allocates nothing: the element-local residual lives in a
 * 32 MiB array inside the library that every GPU loading the library holds
 * until exit.  Meshes needing more (E * P * c * sizeof(real) > 32 MiB) are
 * rejected with SALVUS_E_INVALID.  All calls share that array (and a status
 * word beside it): calls that overlap on the GPU race and must be serialised
 * by the caller.  The first call on a device looks up the array's device
 * address; make it before any stream capture.  FP64 calls on meshes created
 * with SALVUS_MESH_FP32_ONLY return SALVUS_E_STATE; fluid-solid
 * (SALVUS_COUPLED2D) meshes return SALVUS_E_UNSUPPORTED, because their
 * coupling terms act on the velocity field, which this call does not take.
 * On meshes whose FP32 stiffness kernel has bounded device waits (tensor-core
 * tetrahedra and triangles) the call synchronises the stream and returns
 * SALVUS_E_TIMEOUT if a wait gave up; otherwise it returns once the work is
 * queued.  The caller's current device is unchanged on return. */
int salvus_apply_stiffness_noalloc(const salvus_mesh *mesh, int32_t precision, const void *u,
                                   void *a, void *stream);

/* ---- problem groups: many meshes of uneven size advanced together ----
 * A group of FP32 single-shot problems of one element class (acoustic quads
 * or elastic hexahedra of one order, on one device) advances with one launch
 * per step stage for all members (SALVUS_GROUP_STEP=persistent: one
 * persistent work-queue launch per step; SALVUS_GROUP_STEP=partitioned: one
 * cooperative launch per step, each member on its own range of resident
 * CTAs): every CTA runs the single-problem
 * kernel body on its member's arrays, so each member's result is bitwise the
 * one it gets alone.  salvus_group_run(g, n) advances
 * every member n steps (graph-replayed in chunks of 32); it orders itself
 * after the members' pending work and their later work after it.  Members
 * stay owned by the caller and must outlive the group; do not advance a
 * member on its own while a group run is in flight.  No reference
 * counterpart (the reference steps one mesh per process, Main.cpp:45-66). */
typedef struct salvus_group salvus_group;
int salvus_group_create(salvus_problem *const *members, int32_t n_members, salvus_group **out);
int salvus_group_run(salvus_group *g, int64_t n_steps);
int salvus_group_synchronize(salvus_group *g);
/* Bound of the device waits of the single-launch group forms
 * (SALVUS_GROUP_STEP=persistent / partitioned), as
 * salvus_problem_set_wait_limit; salvus_group_synchronize then reports
 * SALVUS_E_TIMEOUT.  salvus_group_clear_status resets the group's and its
 * members' status words (set the members' fields again before continuing). */
int salvus_group_set_wait_limit(salvus_group *g, int64_t cycles);
int salvus_group_clear_status(salvus_group *g);
int salvus_group_destroy(salvus_group *g);

/* ---- serving: continuous batching of forward-modelling jobs ----
 * No reference counterpart (the reference runs one simulation per process,
 * Main.cpp:10-78).  A server owns one GPU and a device-memory budget.  A
 * scheduler thread admits queued jobs while the budget and the running-job
 * limit allow, prepares them on a worker thread (mesh flattening overlaps the
 * GPU work of running jobs), advances every running job in graph-replayed
 * chunks of steps on its own stream so their kernels overlap on the device,
 * copies each chunk's seismogram samples to the host as it completes, and
 * frees a job's device memory when it finishes.  Jobs never share device
 * state, so a job's result is the same alone and in any mix. */
typedef struct {
  salvus_mesh_desc mesh; /* copied at submit */
  int32_t precision;     /* SALVUS_FP32 or SALVUS_FP64 */
  int32_t n_sources;
  const salvus_source *sources;
  int32_t n_receivers;
  int32_t reserved;
  const double *receivers; /* [n_receivers][3] */
  double dt;
  int64_t n_steps;
} salvus_job_desc;

enum salvus_job_state { SALVUS_JOB_QUEUED = 0, SALVUS_JOB_RUNNING = 1, SALVUS_JOB_DONE = 2,
                        SALVUS_JOB_FAILED = 3, SALVUS_JOB_CANCELLED = 4 };

typedef struct {
  int64_t submitted, completed, failed, running, queued;
  double p50_latency_s, p99_latency_s, mean_latency_s;
  double gll_point_updates; /* sum over completed jobs of G * steps */
  double busy_seconds;      /* wall time with at least one job admitted */
  int64_t peak_device_bytes;
  double prep_seconds;      /* sum over jobs of host + device preparation time (worker threads) */
} salvus_server_stats;

typedef struct salvus_server salvus_server;

int salvus_server_create(int device, int64_t memory_budget_bytes, int32_t max_running,
                         int32_t chunk_steps, salvus_server **out);
/* Copies the description (mesh arrays, sources, receivers); the caller's
 * buffers may be reused at once.  Rejects jobs that can never fit the budget. */
int salvus_server_submit(salvus_server *s, const salvus_job_desc *job, int64_t *job_id);
int salvus_server_poll(salvus_server *s, int64_t job_id, int32_t *state, int64_t *steps_done,
                       int64_t *n_nodes);
/* Seismogram samples [receivers][c][count] for steps [first, first+count)
 * already streamed back (count <= steps_done - first). */
int salvus_server_seismograms(salvus_server *s, int64_t job_id, int64_t first, int64_t count,
                              double *out);
/* Blocks until the job is done / failed / cancelled or timeout_s passes
 * (SALVUS_E_TIMEOUT). */
int salvus_server_wait(salvus_server *s, int64_t job_id, double timeout_s);
int salvus_server_cancel(salvus_server *s, int64_t job_id);
/* Drops a finished job's host results. */
int salvus_server_release(salvus_server *s, int64_t job_id);
int salvus_server_stats_read(salvus_server *s, salvus_server_stats *out);
/* Stops the scheduler (running jobs are cancelled) and frees everything. */
int salvus_server_destroy(salvus_server *s);

/* ---- measurement ---- */
/* Device time of the kernels launched by the last salvus_run / salvus_step
 * calls since the last reset, per kernel class (CUDA events on the problem
 * stream): names[i] (static strings), total_ms[i], launches[i].  Profiling
 * adds an event pair per launch; enable only for measurement. */
int salvus_profile_enable(salvus_problem *p, int32_t enable);
int salvus_profile_read(salvus_problem *p, int32_t max_entries, const char **names,
                        double *total_ms, int64_t *launches, int32_t *n_entries);
/* Total kernel launches issued by this library in this process. */
int64_t salvus_launch_count(void);

/* Energy of the current state, 1/2 v^T M v (kinetic) and 1/2 u^T K u
 * (strain, with Dirichlet rows zeroed), each summed in FP64 with Kahan
 * compensation on the GPU and over the CTA partials in a fixed order, so the
 * result is the same on every run.  No counterpart in the reference: a
 * conservation diagnostic (the explicit Newmark step keeps it bounded
 * without sources).  Single-shot problems only.  Synchronous. */
int salvus_problem_energy(salvus_problem *problem, double *kinetic, double *strain);

/* ---- Exodus II meshes and models (no reference-side library needed) ----
 * Reads the NetCDF classic containers (CDF-1, 64-bit-offset CDF-2) that the
 * Exodus library writes, with the Exodus II names the reference reads:
 * Mesh::read (Mesh.cpp:53-86, DMPlexCreateExodusFromFile) and
 * ExodusModel::read (ExodusModel.cpp:37-81): coordinates, element blocks
 * (QUAD4 / HEX8 / TRI3 / TET4, one type), elemental variables of the first
 * time step, side sets.  Cells come back 0-based in this library's vertex
 * orders (HEX8 bottom face reversed, TET4 n0 n2 n1 n3).  NetCDF-4 (HDF5)
 * files are rejected (SALVUS_E_UNSUPPORTED). */
typedef struct salvus_exodus salvus_exodus;
int salvus_exodus_open(const char *path, salvus_exodus **out);
int salvus_exodus_close(salvus_exodus *file);
int salvus_exodus_info(const salvus_exodus *file, int32_t *shape, int32_t *dim,
                       int64_t *n_vertices, int64_t *n_elements, int32_t *n_elem_vars,
                       int32_t *n_side_sets);
/* vertices [n_vertices][dim], cells [n_elements][nv] (either may be NULL) */
int salvus_exodus_mesh(const salvus_exodus *file, double *vertices, int64_t *cells);
int salvus_exodus_variable_name(const salvus_exodus *file, int32_t i, char *buf, int32_t len);
/* elemental variable by name, [n_elements] */
int salvus_exodus_variable(const salvus_exodus *file, const char *name, double *vals);
/* salvus_mesh_desc params for a physics from the per-vertex variables NAME_<i>
 * (ExodusModel::getElementalMaterialParameterAtVertex ExodusModel.cpp:422-470,
 * VP <-> VPV fallback): acoustic VP; elastic3d RHO, VP, VS (VPH / VSH / ETA,
 * when present, must equal VPV / VSV / 1); elastic2d RHO C11 C13 C33 C55;
 * coupled2d the "fluid" flag then VP RHO C11 C13 C33 C55 (absent names 0). */
int salvus_exodus_params(const salvus_exodus *file, int32_t physics, double *params);
/* The reference's six Elastic3D parameters (Elastic3D::attachMaterialProperties,
 * Elastic3D.cpp:33-54), [6][n_elements][nv] RHO VPV VPH VSV VSH ETA, for a
 * mesh created with SALVUS_MESH_ELASTIC_TI: VPV / VSV fall back to VP / VS,
 * VPH / VSH default to VPV / VSV and ETA to 1 when the file lacks them. */
int salvus_exodus_elastic3d_params(const salvus_exodus *file, double *params);
int salvus_exodus_side_set_name(const salvus_exodus *file, int32_t i, char *buf, int32_t len);
/* Global nodes of a mesh built from this file that lie on the named side set
 * (Mesh::setupTopology's "Face Sets", Mesh.cpp:286-312): count first (nodes
 * NULL), then the ascending list.  For salvus_problem_set_dirichlet. */
int salvus_exodus_side_set_nodes(const salvus_exodus *file, const salvus_mesh *mesh,
                                 const char *name, int64_t *count, int64_t *nodes);

#ifdef __cplusplus
}
#endif
#endif
