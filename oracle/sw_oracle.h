/*
 * CPU oracle for the MPAS shallow-water RK4 forward / tangent-linear / adjoint path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of the reference Fortran
 * (src/mpas_sw_dyncore.f90, src/mpas_sw_dyncore_tlm.f90, src/mpas_sw_dyncore_adj.f90,
 * src/mpas_sw_operators.f90, src/mpas_sw_module.f90, src/mpas_sw_testcases.f90), kept in the
 * reference's loop order, scatter order and expression order, built with -O2 -ffp-contract=off.
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg use it; the product
 * library never links or calls it.
 *
 * Parity status: the reference cannot be compiled here (no Fortran compiler), so the oracle is
 * pinned by self-consistency (dot-product test, finite differences, known-answer Williamson
 * TC2) and by golden vectors it generated itself; it is not pinned against reference output.
 *
 * Storage follows the Fortran module exactly: every array is column-major with the reference's
 * dimensions, indices are 1-based, and nVertLevels must be 1.  A module instance is a table of
 * pointers (one per module variable) plus scalar dims/config; the caller owns the memory.
 */
#ifndef SW_ORACLE_H
#define SW_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* real-valued module arrays (src/mpas_sw_module.f90:57-201) */
#define ORC_REALS(X) \
  X(u) X(h) X(tracers) X(u_tl) X(h_tl) X(tracers_tl) X(u_ad) X(h_ad) X(tracers_ad) \
  X(u_src) X(h_s) X(fCell) X(fVertex) X(fEdge) X(areaCell) X(invAreaCell) X(dvEdge) X(dcEdge) \
  X(weightsOnEdge) X(kiteAreasOnVertex) X(meshDensity) X(areaTriangle) \
  X(latCell) X(lonCell) X(xCell) X(yCell) X(zCell) X(meshScalingDel2) X(meshScalingDel4) \
  X(deriv_two) X(latEdge) X(lonEdge) X(xEdge) X(yEdge) X(zEdge) X(angleEdge) \
  X(latVertex) X(lonVertex) X(xVertex) X(yVertex) X(zVertex) X(defc_a) X(defc_b) \
  X(localVerticalUnitVectors) X(edgeNormalVectors) X(cellTangentPlane) X(coeffs_reconstruct) \
  X(uReconstructX) X(uReconstructY) X(uReconstructZ) X(uReconstructZonal) \
  X(uReconstructMeridional) X(v) X(h_edge) X(h_vertex) X(pv_edge) X(pv_vertex) X(pv_cell) \
  X(circulation) X(vorticity) X(divergence) X(ke) X(vh) X(vorticity_cell) X(gradPVn) X(gradPVt) \
  X(uReconstructX_tl) X(uReconstructY_tl) X(uReconstructZ_tl) X(uReconstructZonal_tl) \
  X(uReconstructMeridional_tl) X(v_tl) X(h_edge_tl) X(h_vertex_tl) X(pv_edge_tl) \
  X(pv_vertex_tl) X(pv_cell_tl) X(circulation_tl) X(vorticity_tl) X(divergence_tl) X(ke_tl) \
  X(vh_tl) X(vorticity_cell_tl) X(gradPVn_tl) X(gradPVt_tl) \
  X(uReconstructX_ad) X(uReconstructY_ad) X(uReconstructZ_ad) X(uReconstructZonal_ad) \
  X(uReconstructMeridional_ad) X(v_ad) X(h_edge_ad) X(h_vertex_ad) X(pv_edge_ad) \
  X(pv_vertex_ad) X(pv_cell_ad) X(circulation_ad) X(vorticity_ad) X(divergence_ad) X(ke_ad) \
  X(vh_ad) X(vorticity_cell_ad) X(gradPVn_ad) X(gradPVt_ad) \
  X(tend_u) X(tend_h) X(tend_tracer) X(tend_u_tl) X(tend_h_tl) X(tend_tracer_tl) \
  X(tend_u_ad) X(tend_h_ad) X(tend_tracer_ad)

/* integer module arrays */
#define ORC_INTS(X) \
  X(boundaryCell) X(boundaryEdge) X(advCells) X(cellsOnCell) X(cellsOnEdge) X(cellsOnVertex) \
  X(edgesOnCell) X(edgesOnEdge) X(edgesOnVertex) X(verticesOnCell) X(verticesOnEdge) \
  X(nEdgesOnCell) X(nEdgesOnEdge)

/* integer / logical scalars (logicals as 0/1) */
#define ORC_ISCAL(X) \
  X(nCells) X(nEdges) X(nVertices) X(nVertLevels) X(nTracers) X(maxEdges) X(maxEdges2) \
  X(vertexDegree) X(R3) X(config_test_case) X(config_h_ScaleWithMesh) \
  X(config_thickness_adv_order) X(config_monotonic) X(config_wind_stress) \
  X(config_bottom_drag) X(on_a_sphere) X(is_periodic) X(rk_step) X(config_advect_tracers)

/* real scalars */
#define ORC_RSCAL(X) \
  X(config_dt) X(config_h_mom_eddy_visc2) X(config_h_mom_eddy_visc4) X(config_apvm_upwinding) \
  X(x_period) X(y_period) X(LHS) X(RHS) X(pt) X(sphere_radius)

#define ORC_ENUM(n) ORC_R_##n,
enum { ORC_REALS(ORC_ENUM) ORC_NREAL };
#undef ORC_ENUM
#define ORC_ENUM(n) ORC_I_##n,
enum { ORC_INTS(ORC_ENUM) ORC_NINT };
#undef ORC_ENUM
#define ORC_ENUM(n) ORC_IS_##n,
enum { ORC_ISCAL(ORC_ENUM) ORC_NISCAL };
#undef ORC_ENUM
#define ORC_ENUM(n) ORC_RS_##n,
enum { ORC_RSCAL(ORC_ENUM) ORC_NRSCAL };
#undef ORC_ENUM

typedef struct {
  double *r[ORC_NREAL];
  int *i[ORC_NINT];
  int is[ORC_NISCAL];
  double rs[ORC_NRSCAL];
} orc_mod;

/* name tables so the host wrapper can bind by name */
int orc_count(int kind);                 /* 0 reals, 1 ints, 2 int scalars, 3 real scalars */
const char *orc_name(int kind, int idx);

/* module subroutines (src/mpas_sw_module.f90:495-1218, src/mpas_sw_testcases.f90) */
int orc_sw_mpas_init_block(orc_mod *m);
int orc_sw_rk4(orc_mod *m);
int orc_sw_rk4_tlm(orc_mod *m);
int orc_sw_rk4_adj(orc_mod *m);
int orc_link_tlm_adj(orc_mod *m, int print);
int orc_sw_test_case_1(orc_mod *m);
int orc_sw_test_case_2(orc_mod *m);
int orc_sw_test_case_5(orc_mod *m);
int orc_sw_test_case_6(orc_mod *m);

/* single stencil calls on the module's current level-1 state (for per-call parity) */
int orc_solve_diagnostics(orc_mod *m);    /* diag(h(1),u(1)) into the module diag arrays */
int orc_compute_tend(orc_mod *m);         /* tend(h(1),u(1)) from the module diag arrays */
int orc_solve_diagnostics_tlm(orc_mod *m);
int orc_compute_tend_tlm(orc_mod *m);
int orc_solve_diagnostics_adj(orc_mod *m);/* consumes module diag _ad, accumulates h_ad(1),u_ad(1) */
int orc_compute_tend_adj(orc_mod *m);     /* consumes tend_*_ad, accumulates into module _ad */
int orc_reconstruct_2d(orc_mod *m);
int orc_compute_scalar_tend(orc_mod *m); /* tend_tracer(tracers(1), u(1), module h_edge) */

#ifdef __cplusplus
}
#endif
#endif
