/*
 * oracle.h -- FP64 CPU restatement of the Salvus explicit spectral-element time
 * step.  TEST INFRASTRUCTURE ONLY: this library is the checker for the CUDA
 * product path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs may load it; the product never links or calls it.
 *
 * Every routine restates the reference algorithm from the cited reference
 * source lines (paths relative to the reference project root).  Node
 * numbering deliberately uses a different method (coordinate keys) from the
 * product (topological keys) so the two implementations share no code.
 */
#ifndef SALVUS_ORACLE_H
#define SALVUS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ORC_TRI / ORC_TET: the P3 mass-lumped simplices (12-node triangle,
 * 50-node tetrahedron) of Triangle.cpp / Tetrahedra.cpp, order 3 only. */
enum { ORC_QUAD = 0, ORC_HEX = 1, ORC_TRI = 2, ORC_TET = 3 };
/* ORC_ELASTIC2D: Elastic2D on quads (Elastic2D.cpp:29-127).
 * ORC_COUPLED2D: quads of both kinds in one mesh, fluid (Scalar) and solid
 * (Elastic2D) per element, coupled across shared edges by the
 * ElasticToAcoustic2D / AcousticToElastic2D surface integrals
 * (ElasticToAcoustic.cpp:26-41, AcousticToElastic2D.cpp:48-60); fields per
 * node [u, ux, uy]. */
enum { ORC_ACOUSTIC = 0, ORC_ELASTIC3D = 1, ORC_ELASTIC2D = 2, ORC_COUPLED2D = 3 };

/* Reference quirk switches ("reference-literal" mode).  The default (0) is the
 * corrected physics that the GPU path is checked against. */
enum {
  /* Order2Newmark.cpp:93-96 lists {"ax","ay","ax","a"}: uz never advances. */
  ORC_Q1_Z_NOT_ADVANCED = 1u << 0,
  /* Elastic3D.cpp:126-133 omits applyTestAndIntegrate on the source term. */
  ORC_Q2_ELASTIC_SRC_UNSCALED = 1u << 1,
  /* TensorQuad.cpp:383-390 applies J^-1 at the output point (not per
   * quadrature point) in the 2-D gradient-test integral. */
  ORC_Q3_QUAD_INVJ_AT_OUTPUT = 1u << 2,
  /* QuadP1.h:20-27,85-86 evaluates dN/dr with r and dN/ds with s swapped
   * (exact only on parallelograms). */
  ORC_Q17_QUAD_SWAPPED_JAC = 1u << 3,
  /* Scalar.cpp:45 / TensorQuad.cpp:194,385 / Hexahedra.cpp:600,702: rebuild
   * the Jacobian and re-interpolate material at every GLL point every call
   * (reference operation count; used for the faithful CPU timing). */
  ORC_FAITHFUL_RECOMPUTE = 1u << 4,
  /* Fluid-solid coupling (ORC_COUPLED2D).  The default restates the
   * reference's coupling exactly; these switches make it consistent, one
   * defect at a time (the consistent velocity-coupled scheme is unstable
   * under the explicit Newmark step, see the oracle tests):
   * K1: Order2Newmark.cpp:38-52 sums every element's mass (fluid 1, solid
   *     rho) into one "mi" shared by u, ux and uy; K1 keeps the fluid mass
   *     for u and the solid mass for ux, uy. */
  ORC_K1_SPLIT_MASS = 1u << 5,
  /* K2: AcousticToElastic2D.cpp:53-58 adds -rho0 int(phi v) to both ax and
   *     ay; K2 multiplies by the fluid's outward normal component. */
  ORC_K2_SOLID_NORMAL = 1u << 6,
  /* K3: ElasticToAcoustic.cpp:17-22 couples a fluid element on every edge
   *     with a neighbour, fluid neighbours included; K3 keeps solid ones. */
  ORC_K3_INTERFACE_EDGES = 1u << 7,
  /* K4: ElasticToAcoustic.cpp:33-37 integrates v_s . n without the vp^2 of
   *     the fluid's natural boundary term (Scalar.cpp:42-55); K4 adds it. */
  ORC_K4_FLUID_VP2 = 1u << 8,
};

typedef struct {
  int shape;             /* ORC_QUAD or ORC_HEX */
  int order;             /* polynomial order N (n = N + 1 GLL points per dim) */
  int physics;           /* ORC_ACOUSTIC or ORC_ELASTIC3D */
  int64_t n_vertices;
  const double *vertices;   /* [n_vertices][dim] */
  int64_t n_elements;
  const int64_t *cells;     /* [n_elements][4 | 8 | 3 | 4]: PETSc right-hand
                               order for quads / hexes, TriP1 / TetP1 vertex
                               order (positively oriented) for simplices */
  /* Per element, per element-vertex material (ExodusModel NAME_0..NAME_k
   * convention, ExodusModel.cpp:455-470):
   *   acoustic: [1][n_elements][nv] = VP
   *   elastic : [6][n_elements][nv] = RHO, VPV, VPH, VSV, VSH, ETA
   *   elastic2d: [5][n_elements][nv] = RHO, C11, C13, C33, C55
   *   coupled2d: [7][n_elements][nv] = FLUID (1 fluid, 0 solid), VP, RHO,
   *              C11, C13, C33, C55 (fluid elements use VP and RHO, solid
   *              elements RHO and C..) */
  const double *params;
  unsigned flags;
  int threads;              /* OpenMP threads for element loops (>=1) */
} orc_desc;

typedef struct orc_problem orc_problem;

/* ---- GLL / Lagrange tables (math restatement of the sympy code generator,
 * src/py/pysalvus/code_generation/quadrature_points_weights.py:55-93,
 * code_generator.py:13-43) ---- */
int orc_gll(int order, double *points, double *weights);
int orc_deriv_matrix(int order, double *D /* [n][n], D[i*n+j] = l_j'(xi_i) */);
int orc_lagrange(int order, double xi, double *l /* [n] */, double *dl /* [n] or NULL */);
double orc_ricker(double t, double f0, double t0, double amp);

/* ---- P3 simplex tables (restatement of the sympy generators
 * src/py/pysalvus/code_generation/triangle_points_weights_polys.py and
 * tetrahedra_points_weights_polys.py + BuildNodesTetrahedraP3.py):
 * nodes [P][3] (unused coordinates 0), weights [P],
 * D[k][i][q] = d phi_i / d xi_k at node q (k < dim). ---- */
int orc_simplex_tables(int shape, double *nodes, double *weights, double *D);
/* phi_i(ref) [P] and d phi_i / d xi_k (ref) as dphi[i][k] (NULL to skip). */
int orc_simplex_basis(int shape, const double *ref, double *phi, double *dphi);

/* ---- element level (single element, no mesh) ---- */
int orc_p1_jacobian(int shape, const double *vtx, const double *ref, unsigned flags,
                    double *detJ, double *invJ /* [d][d] */);
int orc_p1_interpolate(int shape, const double *ref, double *w /* [4|8] */);
int orc_check_hull(int shape, const double *vtx, const double *x);
int orc_inverse_map(int shape, const double *vtx, const double *x, double *ref);
/* grad[p][d] of nodal field u[p] (computeGradient). */
int orc_element_gradient(int shape, int order, const double *vtx, unsigned flags,
                         const double *u, double *grad);
/* out[p] = integral of grad(phi_p) . f (applyGradTestAndIntegrate). */
int orc_element_grad_test(int shape, int order, const double *vtx, unsigned flags,
                          const double *f /* [P][d] */, double *out);
/* out[p] = f[p] w_p detJ_p (applyTestAndIntegrate). */
int orc_element_test(int shape, int order, const double *vtx, unsigned flags,
                     const double *f, double *out);
/* delta-function coefficients l_p(ref)/(w_p detJ_p) (getDeltaFunctionCoefficients). */
int orc_element_delta(int shape, int order, const double *vtx, unsigned flags,
                      const double *ref, double *out);
/* P1 vertex parameter interpolated to GLL points (ParAtIntPts). */
int orc_element_par(int shape, int order, const double *par_vtx, double *out);

/* ---- problem level ---- */
orc_problem *orc_create(const orc_desc *d);
void orc_destroy(orc_problem *p);
const char *orc_last_error(void);
int64_t orc_num_nodes(const orc_problem *p);
int orc_num_components(const orc_problem *p);
int orc_node_coords(const orc_problem *p, double *xyz /* [G][dim] */);
/* kind 0: force, comp = direction [c]; kind 1: moment tensor
 * comp = [Mxx, Myy, Mzz, Myz, Mxz, Mxy] (3-D) or [Mxx, Myy, Mxy] (2-D).
 * Returns source index or <0. */
int orc_add_source(orc_problem *p, const double *x, double f0, double t0, double amp,
                   int kind, const double *comp);
int orc_add_receiver(orc_problem *p, const double *x);
/* Homogeneous Dirichlet (HomogeneousDirichlet.cpp:65-73): zero the element
 * stiffness rows of every element point on these nodes (oracle numbering). */
int orc_set_dirichlet(orc_problem *p, int64_t n, const int64_t *nodes);
/* which: 0 = u, 1 = v.  Arrays are [G][c]. */
int orc_set_field(orc_problem *p, int which, const double *vals);
int orc_get_field(const orc_problem *p, int which, double *vals);
int orc_inverse_mass(const orc_problem *p, double *mi /* [G] */);
/* Per-component inverse mass [G][c] (coupled meshes: fluid u and solid ux,
 * uy carry separate masses; 0 where a component has no mass). */
int orc_inverse_mass_c(const orc_problem *p, double *mi);
/* -K u (no sources, no coupling) for a given u [G][c]. */
int orc_apply_stiffness(orc_problem *p, const double *u, double *ku);
/* Advance nsteps (Main.cpp:45-66 loop body).  seis may be NULL, else
 * [n_receivers][c][nsteps] of u sampled after each step. */
int orc_run(orc_problem *p, int64_t nsteps, double dt, double *seis);
/* a = M^-1 (f(t) - K u) for the current state, [G][c]. */
int orc_acceleration(orc_problem *p, double t, double *a);
/* lambda_max of M^-1 K by power iteration (dt_crit = 2/sqrt(lambda)). */
double orc_max_eigenvalue(orc_problem *p, int iters, uint64_t seed);
/* Kinetic + strain energy 0.5 v^T M v + 0.5 u^T K u (FP64, fixed order). */
double orc_energy(orc_problem *p);
int64_t orc_step_index(const orc_problem *p);

#ifdef __cplusplus
}
#endif
#endif
