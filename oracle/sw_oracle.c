/*
 * CPU oracle (TEST INFRASTRUCTURE ONLY) — FP64 restatement of the reference Fortran.
 * See sw_oracle.h for scope, storage conventions and parity status.  Each routine cites the
 * reference routine it restates; loop order, scatter order and the left-to-right evaluation of
 * every expression follow the Fortran, so with -ffp-contract=off the results are those of the
 * f2py build (-fdefault-real-8, no FMA) up to libm differences in sin/cos/sqrt/pow.
 */
#include "sw_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* 1-based, column-major accessors */
#define A1(p, i) ((p)[(i) - 1])
#define A2(p, ld, i, j) ((p)[((i) - 1) + (size_t)(ld) * ((j) - 1)])
#define A3(p, l1, l2, i, j, k) ((p)[((i) - 1) + (size_t)(l1) * (((j) - 1) + (size_t)(l2) * ((k) - 1))])

#define GRAVITY 9.80616                  /* src/mpas_sw_dyncore.f90:414 */
#define RHO_REF 1000.0                   /* src/mpas_sw_dyncore.f90:460 */
#define PII 3.141592653589793            /* src/mpas_sw_module.f90:8 */
#define A_EARTH 6371229.0                /* src/mpas_sw_module.f90:9 */
#define OMEGA 7.29212e-5                 /* src/mpas_sw_module.f90:10 */

static const char *real_names[] = {
#define ORC_NAME(n) #n,
    ORC_REALS(ORC_NAME)
};
static const char *int_names[] = {ORC_INTS(ORC_NAME)};
static const char *iscal_names[] = {ORC_ISCAL(ORC_NAME)};
static const char *rscal_names[] = {ORC_RSCAL(ORC_NAME)};
#undef ORC_NAME

int orc_count(int kind) {
  switch (kind) {
    case 0: return ORC_NREAL;
    case 1: return ORC_NINT;
    case 2: return ORC_NISCAL;
    case 3: return ORC_NRSCAL;
  }
  return -1;
}

const char *orc_name(int kind, int idx) {
  if (idx < 0 || idx >= orc_count(kind)) return NULL;
  switch (kind) {
    case 0: return real_names[idx];
    case 1: return int_names[idx];
    case 2: return iscal_names[idx];
    case 3: return rscal_names[idx];
  }
  return NULL;
}

#define R(n) (m->r[ORC_R_##n])
#define I(n) (m->i[ORC_I_##n])
#define IS(n) (m->is[ORC_IS_##n])
#define RS(n) (m->rs[ORC_RS_##n])

static double *dalloc(size_t n) {
  double *p = (double *)calloc(n ? n : 1, sizeof(double));
  if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
  return p;
}

/* ---------------------------------------------------------------------------------------- */
/* Forward diagnostics: src/mpas_sw_dyncore.f90:1-361 (sw_compute_solve_diagnostics)        */
/* ---------------------------------------------------------------------------------------- */
static void diag_fwd(orc_mod *m, double dt, const double *h, const double *u, double *v,
                     double *h_edge, double *h_vertex, double *circulation, double *vorticity,
                     double *divergence, double *ke, double *pv_edge, double *pv_vertex,
                     double *pv_cell, double *vorticity_cell, double *gradPVn, double *gradPVt) {
  const int nCells = IS(nCells), nEdges = IS(nEdges), nVertices = IS(nVertices);
  const int maxEdges = IS(maxEdges), maxEdges2 = IS(maxEdges2), vertexDegree = IS(vertexDegree);
  const int *cellsOnEdge = I(cellsOnEdge), *verticesOnEdge = I(verticesOnEdge);
  const int *edgesOnCell = I(edgesOnCell), *edgesOnEdge = I(edgesOnEdge);
  const int *edgesOnVertex = I(edgesOnVertex), *cellsOnVertex = I(cellsOnVertex);
  const int *nEdgesOnCell = I(nEdgesOnCell), *nEdgesOnEdge = I(nEdgesOnEdge);
  const int *cellsOnCell = I(cellsOnCell), *boundaryEdge = I(boundaryEdge);
  int *boundaryCell = I(boundaryCell);
  const double *dcEdge = R(dcEdge), *dvEdge = R(dvEdge), *areaCell = R(areaCell);
  const double *areaTriangle = R(areaTriangle), *fVertex = R(fVertex);
  const double *weightsOnEdge = R(weightsOnEdge), *kiteAreasOnVertex = R(kiteAreasOnVertex);
  const double *deriv_two = R(deriv_two);
  const double apvm = RS(config_apvm_upwinding);
  const int order = IS(config_thickness_adv_order);
  int iEdge, iCell, iVertex, i, cell1, cell2, eoe;
  double r, coef_3rd_order, d2fdx2_cell1, d2fdx2_cell2;

  /* :77-87 */
  for (iCell = 1; iCell <= nCells; iCell++) A1(boundaryCell, iCell) = 0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    if (A1(boundaryEdge, iEdge) == 1) {
      A1(boundaryCell, A2(cellsOnEdge, 2, 1, iEdge)) = 1;
      A1(boundaryCell, A2(cellsOnEdge, 2, 2, iEdge)) = 1;
    }
  }
  /* :91-93 */
  coef_3rd_order = 0.;
  if (order == 3) coef_3rd_order = 1.0;
  if (order == 3 && IS(config_monotonic)) coef_3rd_order = 0.25;

  if (order == 2) { /* :95-105 */
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge);
      cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      if (cell1 <= nCells && cell2 <= nCells)
        A1(h_edge, iEdge) = 0.5 * (A1(h, cell1) + A1(h, cell2));
    }
  } else if (order == 3 || order == 4) { /* :107-199 */
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge);
      cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      if (cell1 <= nCells && cell2 <= nCells) {
        d2fdx2_cell1 = 0.0;
        d2fdx2_cell2 = 0.0;
        if (A1(boundaryCell, cell1) == 0 && A1(boundaryCell, cell2) == 0) {
          d2fdx2_cell1 = A3(deriv_two, 15, 2, 1, 1, iEdge) * A1(h, cell1);
          d2fdx2_cell2 = A3(deriv_two, 15, 2, 1, 2, iEdge) * A1(h, cell2);
          for (i = 1; i <= A1(nEdgesOnCell, cell1); i++)
            d2fdx2_cell1 = d2fdx2_cell1 + A3(deriv_two, 15, 2, i + 1, 1, iEdge) *
                                              A1(h, A2(cellsOnCell, maxEdges, i, cell1));
          for (i = 1; i <= A1(nEdgesOnCell, cell2); i++)
            d2fdx2_cell2 = d2fdx2_cell2 + A3(deriv_two, 15, 2, i + 1, 2, iEdge) *
                                              A1(h, A2(cellsOnCell, maxEdges, i, cell2));
        }
        const double dc2 = A1(dcEdge, iEdge) * A1(dcEdge, iEdge);
        if (order == 3) {
          if (A1(u, iEdge) > 0)
            A1(h_edge, iEdge) = 0.5 * (A1(h, cell1) + A1(h, cell2)) -
                                dc2 * (d2fdx2_cell1 + d2fdx2_cell2) / 12. -
                                dc2 * coef_3rd_order * (d2fdx2_cell1 - d2fdx2_cell2) / 12.;
          else
            A1(h_edge, iEdge) = 0.5 * (A1(h, cell1) + A1(h, cell2)) -
                                dc2 * (d2fdx2_cell1 + d2fdx2_cell2) / 12. +
                                dc2 * coef_3rd_order * (d2fdx2_cell1 - d2fdx2_cell2) / 12.;
        } else {
          A1(h_edge, iEdge) = 0.5 * (A1(h, cell1) + A1(h, cell2)) -
                              dc2 * (d2fdx2_cell1 + d2fdx2_cell2) / 12.;
        }
      }
    }
  }

  /* circulation and vorticity :208-219 */
  for (iVertex = 1; iVertex <= nVertices; iVertex++) A1(circulation, iVertex) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    const int v1 = A2(verticesOnEdge, 2, 1, iEdge), v2 = A2(verticesOnEdge, 2, 2, iEdge);
    A1(circulation, v1) = A1(circulation, v1) - A1(dcEdge, iEdge) * A1(u, iEdge);
    A1(circulation, v2) = A1(circulation, v2) + A1(dcEdge, iEdge) * A1(u, iEdge);
  }
  for (iVertex = 1; iVertex <= nVertices; iVertex++)
    A1(vorticity, iVertex) = A1(circulation, iVertex) / A1(areaTriangle, iVertex);

  /* divergence :222-242 */
  for (iCell = 1; iCell <= nCells; iCell++) A1(divergence, iCell) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge);
    cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    if (cell1 <= nCells)
      A1(divergence, cell1) = A1(divergence, cell1) + A1(u, iEdge) * A1(dvEdge, iEdge);
    if (cell2 <= nCells)
      A1(divergence, cell2) = A1(divergence, cell2) - A1(u, iEdge) * A1(dvEdge, iEdge);
  }
  for (iCell = 1; iCell <= nCells; iCell++) {
    r = 1.0 / A1(areaCell, iCell);
    A1(divergence, iCell) = A1(divergence, iCell) * r;
  }

  /* kinetic energy :245-256 */
  for (iCell = 1; iCell <= nCells; iCell++) A1(ke, iCell) = 0.0;
  for (iCell = 1; iCell <= nCells; iCell++) {
    for (i = 1; i <= A1(nEdgesOnCell, iCell); i++) {
      iEdge = A2(edgesOnCell, maxEdges, i, iCell);
      A1(ke, iCell) = A1(ke, iCell) + 0.25 * A1(dcEdge, iEdge) * A1(dvEdge, iEdge) *
                                          (A1(u, iEdge) * A1(u, iEdge));
    }
    A1(ke, iCell) = A1(ke, iCell) / A1(areaCell, iCell);
  }

  /* tangential velocity :259-267 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(v, iEdge) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    for (i = 1; i <= A1(nEdgesOnEdge, iEdge); i++) {
      eoe = A2(edgesOnEdge, maxEdges2, i, iEdge);
      A1(v, iEdge) = A1(v, iEdge) + A2(weightsOnEdge, maxEdges2, i, iEdge) * A1(u, eoe);
    }
  }

  /* h_vertex, pv_vertex :282-292 */
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    A1(h_vertex, iVertex) = 0.0;
    for (i = 1; i <= vertexDegree; i++)
      A1(h_vertex, iVertex) = A1(h_vertex, iVertex) +
                              A1(h, A2(cellsOnVertex, vertexDegree, i, iVertex)) *
                                  A2(kiteAreasOnVertex, vertexDegree, i, iVertex);
    A1(h_vertex, iVertex) = A1(h_vertex, iVertex) / A1(areaTriangle, iVertex);
    A1(pv_vertex, iVertex) = (A1(fVertex, iVertex) + A1(vorticity, iVertex)) / A1(h_vertex, iVertex);
  }

  /* gradPVt :296-301 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++)
    A1(gradPVt, iEdge) = (A1(pv_vertex, A2(verticesOnEdge, 2, 2, iEdge)) -
                          A1(pv_vertex, A2(verticesOnEdge, 2, 1, iEdge))) / A1(dvEdge, iEdge);

  /* pv_edge :305-313 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(pv_edge, iEdge) = 0.0;
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    for (i = 1; i <= vertexDegree; i++) {
      iEdge = A2(edgesOnVertex, vertexDegree, i, iVertex);
      A1(pv_edge, iEdge) = A1(pv_edge, iEdge) + 0.5 * A1(pv_vertex, iVertex);
    }
  }
  /* APVM tangential :316-320 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++)
    A1(pv_edge, iEdge) = A1(pv_edge, iEdge) - apvm * A1(v, iEdge) * dt * A1(gradPVt, iEdge);

  /* pv_cell, vorticity_cell :324-340 */
  for (iCell = 1; iCell <= nCells; iCell++) {
    A1(pv_cell, iCell) = 0.0;
    A1(vorticity_cell, iCell) = 0.0;
  }
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    for (i = 1; i <= vertexDegree; i++) {
      iCell = A2(cellsOnVertex, vertexDegree, i, iVertex);
      if (iCell <= nCells) {
        A1(pv_cell, iCell) = A1(pv_cell, iCell) + A2(kiteAreasOnVertex, vertexDegree, i, iVertex) *
                                                      A1(pv_vertex, iVertex) / A1(areaCell, iCell);
        A1(vorticity_cell, iCell) = A1(vorticity_cell, iCell) +
                                    A2(kiteAreasOnVertex, vertexDegree, i, iVertex) *
                                        A1(vorticity, iVertex) / A1(areaCell, iCell);
      }
    }
  }

  /* gradPVn :344-352 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(gradPVn, iEdge) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    if (A2(cellsOnEdge, 2, 1, iEdge) <= nCells && A2(cellsOnEdge, 2, 2, iEdge) <= nCells)
      A1(gradPVn, iEdge) = (A1(pv_cell, A2(cellsOnEdge, 2, 2, iEdge)) -
                            A1(pv_cell, A2(cellsOnEdge, 2, 1, iEdge))) / A1(dcEdge, iEdge);
  }
  /* APVM normal :355-359 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++)
    A1(pv_edge, iEdge) = A1(pv_edge, iEdge) - apvm * A1(u, iEdge) * dt * A1(gradPVn, iEdge);
}

/* compute_mesh_scaling: src/mpas_sw_dyncore.f90:363-393 */
static void mesh_scaling(orc_mod *m) {
  const int nEdges = IS(nEdges);
  for (int iEdge = 1; iEdge <= nEdges; iEdge++) {
    A1(R(meshScalingDel2), iEdge) = 1.0;
    A1(R(meshScalingDel4), iEdge) = 1.0;
  }
  if (IS(config_h_ScaleWithMesh)) {
    for (int iEdge = 1; iEdge <= nEdges; iEdge++) {
      const int cell1 = A2(I(cellsOnEdge), 2, 1, iEdge), cell2 = A2(I(cellsOnEdge), 2, 2, iEdge);
      const double md = (A1(R(meshDensity), cell1) + A1(R(meshDensity), cell2)) / 2.0;
      A1(R(meshScalingDel2), iEdge) = 1.0 / pow(md, 5.0 / 12.0);
      A1(R(meshScalingDel4), iEdge) = 1.0 / pow(md, 5.0 / 6.0);
    }
  }
}

/* ---------------------------------------------------------------------------------------- */
/* Forward tendencies: src/mpas_sw_dyncore.f90:395-639 (sw_compute_tend)                      */
/* ---------------------------------------------------------------------------------------- */
static void tend_fwd(orc_mod *m, const double *h, const double *u, const double *h_edge,
                     const double *vorticity, const double *divergence, const double *ke,
                     const double *pv_edge, double *tend_h, double *tend_u) {
  const int nCells = IS(nCells), nEdges = IS(nEdges), nVertices = IS(nVertices);
  const int maxEdges2 = IS(maxEdges2);
  const int *cellsOnEdge = I(cellsOnEdge), *verticesOnEdge = I(verticesOnEdge);
  const int *edgesOnEdge = I(edgesOnEdge), *nEdgesOnEdge = I(nEdgesOnEdge);
  const double *dcEdge = R(dcEdge), *dvEdge = R(dvEdge), *areaCell = R(areaCell);
  const double *areaTriangle = R(areaTriangle), *h_s = R(h_s), *u_src = R(u_src);
  const double *weightsOnEdge = R(weightsOnEdge);
  const double *sc2 = R(meshScalingDel2), *sc4 = R(meshScalingDel4);
  const double visc2 = RS(config_h_mom_eddy_visc2), visc4 = RS(config_h_mom_eddy_visc4);
  int iEdge, iCell, iVertex, j, cell1, cell2, vertex1, vertex2, eoe;
  double flux, q, workpv, r, u_diffusion, ke_edge;

  /* :468-482 */
  for (iCell = 1; iCell <= nCells; iCell++) A1(tend_h, iCell) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge);
    cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    flux = A1(u, iEdge) * A1(dvEdge, iEdge) * A1(h_edge, iEdge);
    A1(tend_h, cell1) = A1(tend_h, cell1) - flux;
    A1(tend_h, cell2) = A1(tend_h, cell2) + flux;
  }
  for (iCell = 1; iCell <= nCells; iCell++) A1(tend_h, iCell) = A1(tend_h, iCell) / A1(areaCell, iCell);

  /* :485-505 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(tend_u, iEdge) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge);
    cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    q = 0.0;
    for (j = 1; j <= A1(nEdgesOnEdge, iEdge); j++) {
      eoe = A2(edgesOnEdge, maxEdges2, j, iEdge);
      workpv = 0.5 * (A1(pv_edge, iEdge) + A1(pv_edge, eoe));
      q = q + A2(weightsOnEdge, maxEdges2, j, iEdge) * A1(u, eoe) * workpv * A1(h_edge, eoe);
    }
    A1(tend_u, iEdge) = q - (A1(ke, cell2) - A1(ke, cell1) +
                             GRAVITY * (A1(h, cell2) + A1(h_s, cell2) - A1(h, cell1) - A1(h_s, cell1))) /
                                A1(dcEdge, iEdge);
  }

  /* del2 :510-524 */
  if (visc2 > 0.0) {
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge);
      cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge);
      vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      u_diffusion = (A1(divergence, cell2) - A1(divergence, cell1)) / A1(dcEdge, iEdge) -
                    (A1(vorticity, vertex2) - A1(vorticity, vertex1)) / A1(dvEdge, iEdge);
      u_diffusion = A1(sc2, iEdge) * visc2 * u_diffusion;
      A1(tend_u, iEdge) = A1(tend_u, iEdge) + u_diffusion;
    }
  }

  /* del4 :530-617 */
  if (visc4 > 0.0) {
    double *delsq_divergence = dalloc(nCells + 1), *delsq_u = dalloc(nEdges + 1);
    double *delsq_circulation = dalloc(nVertices + 1), *delsq_vorticity = dalloc(nVertices + 1);
    for (iEdge = 1; iEdge <= nEdges + 1; iEdge++) A1(delsq_u, iEdge) = 0.0;
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge);
      cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge);
      vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      A1(delsq_u, iEdge) = (A1(divergence, cell2) - A1(divergence, cell1)) / A1(dcEdge, iEdge) -
                           (A1(vorticity, vertex2) - A1(vorticity, vertex1)) / A1(dvEdge, iEdge);
    }
    for (iVertex = 1; iVertex <= nVertices + 1; iVertex++) A1(delsq_circulation, iVertex) = 0.0;
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge);
      vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      A1(delsq_circulation, vertex1) = A1(delsq_circulation, vertex1) - A1(dcEdge, iEdge) * A1(delsq_u, iEdge);
      A1(delsq_circulation, vertex2) = A1(delsq_circulation, vertex2) + A1(dcEdge, iEdge) * A1(delsq_u, iEdge);
    }
    for (iVertex = 1; iVertex <= nVertices; iVertex++) {
      r = 1.0 / A1(areaTriangle, iVertex);
      A1(delsq_vorticity, iVertex) = A1(delsq_circulation, iVertex) * r;
    }
    for (iCell = 1; iCell <= nCells + 1; iCell++) A1(delsq_divergence, iCell) = 0.0;
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge);
      cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      A1(delsq_divergence, cell1) = A1(delsq_divergence, cell1) + A1(delsq_u, iEdge) * A1(dvEdge, iEdge);
      A1(delsq_divergence, cell2) = A1(delsq_divergence, cell2) - A1(delsq_u, iEdge) * A1(dvEdge, iEdge);
    }
    for (iCell = 1; iCell <= nCells; iCell++) {
      r = 1.0 / A1(areaCell, iCell);
      A1(delsq_divergence, iCell) = A1(delsq_divergence, iCell) * r;
    }
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge);
      cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge);
      vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      u_diffusion = (A1(delsq_divergence, cell2) - A1(delsq_divergence, cell1)) / A1(dcEdge, iEdge) -
                    (A1(delsq_vorticity, vertex2) - A1(delsq_vorticity, vertex1)) / A1(dvEdge, iEdge);
      u_diffusion = A1(sc4, iEdge) * visc4 * u_diffusion;
      A1(tend_u, iEdge) = A1(tend_u, iEdge) - u_diffusion;
    }
    free(delsq_divergence); free(delsq_u); free(delsq_circulation); free(delsq_vorticity);
  }

  /* wind stress :620-625 */
  if (IS(config_wind_stress)) {
    for (iEdge = 1; iEdge <= nEdges; iEdge++)
      A1(tend_u, iEdge) = A1(tend_u, iEdge) + A1(u_src, iEdge) / RHO_REF / A1(h_edge, iEdge);
  }
  /* bottom drag :627-637 */
  if (IS(config_bottom_drag)) {
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      ke_edge = 0.5 * (A1(ke, A2(cellsOnEdge, 2, 1, iEdge)) + A1(ke, A2(cellsOnEdge, 2, 2, iEdge)));
      A1(tend_u, iEdge) = A1(tend_u, iEdge) -
                          1.0e-3 * A1(u, iEdge) * sqrt(2.0 * ke_edge) / A1(h_edge, iEdge);
    }
  }
}

/* ---------------------------------------------------------------------------------------- */
/* Geometry + RBF reconstruction setup: src/mpas_sw_operators.f90:2-279, 413-625              */
/* ---------------------------------------------------------------------------------------- */
/* Tracer transport, the call the reference leaves out of its RK4 loop
   (src/mpas_sw_module.f90:587, "call sw_compute_scalar_tend() ! omitted"): MPAS's
   sw_compute_scalar_tend at advection order 2 (MPAS-Model shallow-water core, not vendored in
   the reference), restated in the form of this file's thickness tendency (:468-482): the
   h_edge-weighted flux of the edge-mean tracer, scattered to both cells of each edge in edge
   order, divided by areaCell afterwards.  tr and tend are (nTracers, nCells), tracer fastest. */
static void scalar_tend_fwd(orc_mod *m, const double *u, const double *h_edge, const double *tr,
                            double *tend) {
  const int nCells = IS(nCells), nEdges = IS(nEdges), nT = IS(nTracers);
  const int *cellsOnEdge = I(cellsOnEdge);
  const double *dvEdge = R(dvEdge), *areaCell = R(areaCell);
  for (int i = 1; i <= nT * nCells; i++) A1(tend, i) = 0.0;
  for (int iEdge = 1; iEdge <= nEdges; iEdge++) {
    const int cell1 = A2(cellsOnEdge, 2, 1, iEdge), cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    const double flux = A1(u, iEdge) * A1(dvEdge, iEdge) * A1(h_edge, iEdge);
    for (int t = 1; t <= nT; t++) {
      const double tr_edge = 0.5 * (A2(tr, nT, t, cell1) + A2(tr, nT, t, cell2));
      A2(tend, nT, t, cell1) = A2(tend, nT, t, cell1) - flux * tr_edge;
      A2(tend, nT, t, cell2) = A2(tend, nT, t, cell2) + flux * tr_edge;
    }
  }
  for (int iCell = 1; iCell <= nCells; iCell++)
    for (int t = 1; t <= nT; t++) A2(tend, nT, t, iCell) = A2(tend, nT, t, iCell) / A1(areaCell, iCell);
}

static void unit_vec(double *x) { /* :118-127 */
  const double mag = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  x[0] = x[0] / mag; x[1] = x[1] / mag; x[2] = x[2] / mag;
}

static void cross3(const double *p1, const double *p2, double *o) { /* :129-138 */
  o[0] = p1[1] * p2[2] - p1[2] * p2[1];
  o[1] = p1[2] * p2[0] - p1[0] * p2[2];
  o[2] = p1[0] * p2[1] - p1[1] * p2[0];
}

static void initialize_vectors(orc_mod *m) { /* :2-116 (non-periodic sphere/plane) */
  const int nCells = IS(nCells), nEdges = IS(nEdges), maxEdges = IS(maxEdges);
  double *lvu = R(localVerticalUnitVectors), *env = R(edgeNormalVectors), *ctp = R(cellTangentPlane);
  const double *xC = R(xCell), *yC = R(yCell), *zC = R(zCell);
  const double *xE = R(xEdge), *yE = R(yEdge), *zE = R(zEdge);
  for (int i = 0; i < 3 * nEdges; i++) env[i] = 0;
  for (int i = 0; i < 3 * nCells; i++) lvu[i] = 0;
  for (int c = 1; c <= nCells; c++) {
    double *l = &A2(lvu, 3, 1, c);
    if (IS(on_a_sphere)) {
      l[0] = A1(xC, c); l[1] = A1(yC, c); l[2] = A1(zC, c);
      unit_vec(l);
    } else {
      l[0] = 0.; l[1] = 0.; l[2] = 1.;
    }
  }
  for (int e = 1; e <= nEdges; e++) {
    const int c1 = A2(I(cellsOnEdge), 2, 1, e), c2 = A2(I(cellsOnEdge), 2, 2, e);
    double *n = &A2(env, 3, 1, e);
    if (c1 == nCells + 1) {
      n[0] = A1(xC, c2) - A1(xE, e); n[1] = A1(yC, c2) - A1(yE, e); n[2] = A1(zC, c2) - A1(zE, e);
    } else if (c2 == nCells + 1) {
      n[0] = A1(xE, e) - A1(xC, c1); n[1] = A1(yE, e) - A1(yC, c1); n[2] = A1(zE, e) - A1(zC, c1);
    } else {
      n[0] = A1(xC, c2) - A1(xC, c1); n[1] = A1(yC, c2) - A1(yC, c1); n[2] = A1(zC, c2) - A1(zC, c1);
    }
    unit_vec(n);
  }
  for (int c = 1; c <= nCells; c++) {
    const int e = A2(I(edgesOnCell), maxEdges, 1, c);
    const double *rHat = &A2(lvu, 3, 1, c);
    const double *n = &A2(env, 3, 1, e);
    double xh[3], yh[3];
    const double nd = 0.0 + n[0] * rHat[0] + n[1] * rHat[1] + n[2] * rHat[2];
    for (int k = 0; k < 3; k++) xh[k] = n[k] - nd * rHat[k];
    unit_vec(xh);
    cross3(rHat, xh, yh);
    unit_vec(yh);
    for (int k = 0; k < 3; k++) {
      A3(ctp, 3, 2, k + 1, 1, c) = xh[k];
      A3(ctp, 3, 2, k + 1, 2, c) = yh[k];
    }
  }
}

/* elgs: src/mpas_sw_operators.f90:560-625 (partial-pivoting Gaussian elimination) */
static void elgs(double *A, int N, int *indx) {
  double *C = dalloc(N);
  int i, j, k = 1, itmp;
  for (i = 1; i <= N; i++) A1(indx, i) = i;
  for (i = 1; i <= N; i++) {
    double c1 = 0.0;
    for (j = 1; j <= N; j++) c1 = fmax(c1, fabs(A2(A, N, i, j)));
    A1(C, i) = c1;
  }
  for (j = 1; j <= N - 1; j++) {
    double pi1 = 0.0;
    for (i = j; i <= N; i++) {
      const double pi = fabs(A2(A, N, A1(indx, i), j)) / A1(C, A1(indx, i));
      if (pi > pi1) { pi1 = pi; k = i; }
    }
    itmp = A1(indx, j); A1(indx, j) = A1(indx, k); A1(indx, k) = itmp;
    for (i = j + 1; i <= N; i++) {
      const double pj = A2(A, N, A1(indx, i), j) / A2(A, N, A1(indx, j), j);
      A2(A, N, A1(indx, i), j) = pj;
      for (k = j + 1; k <= N; k++)
        A2(A, N, A1(indx, i), k) = A2(A, N, A1(indx, i), k) - pj * A2(A, N, A1(indx, j), k);
    }
  }
  free(C);
}

/* mpas_legs: src/mpas_sw_operators.f90:529-558 */
static void legs(double *A, int N, double *B, double *X, int *indx) {
  elgs(A, N, indx);
  for (int i = 1; i <= N - 1; i++)
    for (int j = i + 1; j <= N; j++)
      A1(B, A1(indx, j)) = A1(B, A1(indx, j)) - A2(A, N, A1(indx, j), i) * A1(B, A1(indx, i));
  A1(X, N) = A1(B, A1(indx, N)) / A2(A, N, A1(indx, N), N);
  for (int i = N - 1; i >= 1; i--) {
    A1(X, i) = A1(B, A1(indx, i));
    for (int j = i + 1; j <= N; j++) A1(X, i) = A1(X, i) - A2(A, N, A1(indx, i), j) * A1(X, j);
    A1(X, i) = A1(X, i) / A2(A, N, A1(indx, i), i);
  }
}

static double evaluate_rbf(double rSquared) { return 1.0 / sqrt(1.0 + rSquared); } /* :519-527 */

/* mpas_rbf_interp_func_3D_plane_vec_const_dir_comp_coeffs + set_up matrix: :413-517 */
static void rbf_coeffs(int n, const double *src /*(n,3)*/, const double *uvec /*(n,3)*/,
                       const double *dest, double alpha, const double *pbv /*(2,3)*/,
                       double *coefficients /*(n,3)*/) {
  const int ms = n + 2;
  double *pts = dalloc(2 * n), *puv = dalloc(2 * n), pdst[2];
  double *matrix = dalloc(ms * ms), *matrixCopy = dalloc(ms * ms), *rhs = dalloc(2 * ms);
  double *coeffs = dalloc(2 * ms);
  int *piv = (int *)calloc(ms, sizeof(int));
  for (int i = 1; i <= n; i++) {
    for (int d = 1; d <= 2; d++) {
      double s = 0.0, t = 0.0;
      for (int k = 1; k <= 3; k++) {
        s = s + A2(src, n, i, k) * A2(pbv, 2, d, k);
        t = t + A2(uvec, n, i, k) * A2(pbv, 2, d, k);
      }
      A2(pts, n, i, d) = s;
      A2(puv, n, i, d) = t;
    }
  }
  for (int d = 1; d <= 2; d++) {
    double s = 0.0;
    for (int k = 1; k <= 3; k++) s = s + dest[k - 1] * A2(pbv, 2, d, k);
    pdst[d - 1] = s;
  }
  /* set_up_vector_dirichlet_rbf_matrix_and_rhs :502-515 */
  for (int j = 1; j <= n; j++) {
    for (int i = j; i <= n; i++) {
      double rs = 0.0, dot = 0.0;
      for (int d = 1; d <= 2; d++) {
        const double df = A2(pts, n, i, d) - A2(pts, n, j, d);
        rs = rs + df * df;
        dot = dot + A2(puv, n, i, d) * A2(puv, n, j, d);
      }
      rs = rs / (alpha * alpha);
      A2(matrix, ms, i, j) = evaluate_rbf(rs) * dot;
      A2(matrix, ms, j, i) = A2(matrix, ms, i, j);
    }
  }
  for (int j = 1; j <= n; j++) {
    double rs = 0.0;
    for (int d = 1; d <= 2; d++) {
      const double df = pdst[d - 1] - A2(pts, n, j, d);
      rs = rs + df * df;
    }
    rs = rs / (alpha * alpha);
    const double rb = evaluate_rbf(rs);
    for (int d = 1; d <= 2; d++) A2(rhs, ms, j, d) = rb * A2(puv, n, j, d);
  }
  for (int i = 1; i <= n; i++) {
    for (int d = 1; d <= 2; d++) {
      A2(matrix, ms, i, n + d) = A2(puv, n, i, d);
      A2(matrix, ms, n + d, i) = A2(matrix, ms, i, n + d);
    }
  }
  A2(rhs, ms, n + 1, 1) = 1.0;
  A2(rhs, ms, n + 2, 2) = 1.0;
  memcpy(matrixCopy, matrix, sizeof(double) * ms * ms);
  legs(matrix, ms, &A2(rhs, ms, 1, 1), &A2(coeffs, ms, 1, 1), piv);
  legs(matrixCopy, ms, &A2(rhs, ms, 1, 2), &A2(coeffs, ms, 1, 2), piv);
  for (int i = 1; i <= 3; i++)
    for (int p = 1; p <= n; p++)
      A2(coefficients, n, p, i) = A2(pbv, 2, 1, i) * A2(coeffs, ms, p, 1) +
                                  A2(pbv, 2, 2, i) * A2(coeffs, ms, p, 2);
  free(pts); free(puv); free(matrix); free(matrixCopy); free(rhs); free(coeffs); free(piv);
}

static void init_reconstruct(orc_mod *m) { /* src/mpas_sw_operators.f90:162-279 (non-periodic) */
  const int nCells = IS(nCells), maxEdges = IS(maxEdges);
  double *cr = R(coeffs_reconstruct);
  for (size_t i = 0; i < (size_t)3 * maxEdges * nCells; i++) cr[i] = 0.0;
  for (int c = 1; c <= nCells; c++) {
    const int n = A1(I(nEdgesOnCell), c);
    double center[3] = {A1(R(xCell), c), A1(R(yCell), c), A1(R(zCell), c)};
    double *loc = dalloc(3 * n), *nrm = dalloc(3 * n), *cw = dalloc(3 * n), tp[6];
    for (int i = 1; i <= n; i++) {
      const int e = A2(I(edgesOnCell), maxEdges, i, c);
      A2(loc, n, i, 1) = A1(R(xEdge), e);
      A2(loc, n, i, 2) = A1(R(yEdge), e);
      A2(loc, n, i, 3) = A1(R(zEdge), e);
      for (int k = 1; k <= 3; k++) A2(nrm, n, i, k) = A2(R(edgeNormalVectors), 3, k, e);
    }
    double alpha = 0.0;
    for (int i = 1; i <= n; i++) {
      double s = 0.0;
      for (int k = 1; k <= 3; k++) {
        const double d = center[k - 1] - A2(loc, n, i, k);
        s = s + d * d;
      }
      alpha = alpha + sqrt(s);
    }
    alpha = alpha / n;
    for (int k = 1; k <= 3; k++) {
      A2(tp, 2, 1, k) = A3(R(cellTangentPlane), 3, 2, k, 1, c);
      A2(tp, 2, 2, k) = A3(R(cellTangentPlane), 3, 2, k, 2, c);
    }
    rbf_coeffs(n, loc, nrm, center, alpha, tp, cw);
    for (int i = 1; i <= n; i++)
      for (int k = 1; k <= 3; k++) A3(cr, 3, maxEdges, k, i, c) = A2(cw, n, i, k);
    free(loc); free(nrm); free(cw);
  }
}

/* mpas_reconstruct_2d: src/mpas_sw_operators.f90:283-370 */
static void reconstruct_fwd(orc_mod *m, const double *u, double *X, double *Y, double *Z,
                            double *Zon, double *Mer) {
  const int nCells = IS(nCells), maxEdges = IS(maxEdges);
  const double *cr = R(coeffs_reconstruct);
  for (int c = 1; c <= nCells; c++) {
    A1(X, c) = 0.0; A1(Y, c) = 0.0; A1(Z, c) = 0.0;
    for (int i = 1; i <= A1(I(nEdgesOnCell), c); i++) {
      const int e = A2(I(edgesOnCell), maxEdges, i, c);
      A1(X, c) = A1(X, c) + A3(cr, 3, maxEdges, 1, i, c) * A1(u, e);
      A1(Y, c) = A1(Y, c) + A3(cr, 3, maxEdges, 2, i, c) * A1(u, e);
      A1(Z, c) = A1(Z, c) + A3(cr, 3, maxEdges, 3, i, c) * A1(u, e);
    }
  }
  if (IS(on_a_sphere)) {
    for (int c = 1; c <= nCells; c++) {
      const double clat = cos(A1(R(latCell), c)), slat = sin(A1(R(latCell), c));
      const double clon = cos(A1(R(lonCell), c)), slon = sin(A1(R(lonCell), c));
      A1(Zon, c) = -A1(X, c) * slon + A1(Y, c) * clon;
      A1(Mer, c) = -(A1(X, c) * clon + A1(Y, c) * slon) * slat + A1(Z, c) * clat;
    }
  } else {
    for (int c = 1; c <= nCells; c++) { A1(Zon, c) = A1(X, c); A1(Mer, c) = A1(Y, c); }
  }
}

/* ---------------------------------------------------------------------------------------- */
/* Tangent linear: src/mpas_sw_dyncore_tlm.f90                                                */
/* ---------------------------------------------------------------------------------------- */
/* sw_compute_solve_diagnostics_tlm :1-447 (order 2 branch; orders 3/4 use deriv_two == 0) */
static void diag_tlm(orc_mod *m, double dt, const double *h, const double *h_tl, const double *u,
                     const double *u_tl) {
  const int nCells = IS(nCells), nEdges = IS(nEdges), nVertices = IS(nVertices);
  const int maxEdges = IS(maxEdges), maxEdges2 = IS(maxEdges2), vertexDegree = IS(vertexDegree);
  const int *cellsOnEdge = I(cellsOnEdge), *verticesOnEdge = I(verticesOnEdge);
  const int *edgesOnCell = I(edgesOnCell), *edgesOnEdge = I(edgesOnEdge);
  const int *edgesOnVertex = I(edgesOnVertex), *cellsOnVertex = I(cellsOnVertex);
  const int *nEdgesOnCell = I(nEdgesOnCell), *nEdgesOnEdge = I(nEdgesOnEdge);
  const double *dcEdge = R(dcEdge), *dvEdge = R(dvEdge), *areaCell = R(areaCell);
  const double *areaTriangle = R(areaTriangle), *fVertex = R(fVertex);
  const double *w = R(weightsOnEdge), *kite = R(kiteAreasOnVertex);
  const double apvm = RS(config_apvm_upwinding);
  double *v = R(v), *v_tl = R(v_tl), *h_edge = R(h_edge), *h_edge_tl = R(h_edge_tl);
  double *h_vertex = R(h_vertex), *h_vertex_tl = R(h_vertex_tl);
  double *circ = R(circulation), *circ_tl = R(circulation_tl);
  double *vort = R(vorticity), *vort_tl = R(vorticity_tl), *div = R(divergence), *div_tl = R(divergence_tl);
  double *ke = R(ke), *ke_tl = R(ke_tl), *pe = R(pv_edge), *pe_tl = R(pv_edge_tl);
  double *pvv = R(pv_vertex), *pvv_tl = R(pv_vertex_tl), *pc = R(pv_cell), *pc_tl = R(pv_cell_tl);
  double *vc = R(vorticity_cell), *vc_tl = R(vorticity_cell_tl);
  double *gpn = R(gradPVn), *gpn_tl = R(gradPVn_tl), *gpt = R(gradPVt), *gpt_tl = R(gradPVt_tl);
  int iEdge, iCell, iVertex, i, cell1, cell2, eoe;
  double r;

  for (iCell = 1; iCell <= nCells; iCell++) A1(I(boundaryCell), iCell) = 0;
  if (IS(config_thickness_adv_order) != 2) {
    /* orders 3/4: with deriv_two == 0 the correction terms vanish; restate generally */
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      double d1 = 0.0, d1t = 0.0, d2 = 0.0, d2t = 0.0;
      const double *dtw = R(deriv_two);
      d1t = A3(dtw, 15, 2, 1, 1, iEdge) * A1(h_tl, cell1);
      d1 = A3(dtw, 15, 2, 1, 1, iEdge) * A1(h, cell1);
      d2t = A3(dtw, 15, 2, 1, 2, iEdge) * A1(h_tl, cell2);
      d2 = A3(dtw, 15, 2, 1, 2, iEdge) * A1(h, cell2);
      for (i = 1; i <= A1(nEdgesOnCell, cell1); i++) {
        d1t = d1t + A3(dtw, 15, 2, i + 1, 1, iEdge) * A1(h_tl, A2(I(cellsOnCell), maxEdges, i, cell1));
        d1 = d1 + A3(dtw, 15, 2, i + 1, 1, iEdge) * A1(h, A2(I(cellsOnCell), maxEdges, i, cell1));
      }
      for (i = 1; i <= A1(nEdgesOnCell, cell2); i++) {
        d2t = d2t + A3(dtw, 15, 2, i + 1, 2, iEdge) * A1(h_tl, A2(I(cellsOnCell), maxEdges, i, cell2));
        d2 = d2 + A3(dtw, 15, 2, i + 1, 2, iEdge) * A1(h, A2(I(cellsOnCell), maxEdges, i, cell2));
      }
      const double dc2 = A1(dcEdge, iEdge) * A1(dcEdge, iEdge);
      double coef = 0.;
      if (IS(config_thickness_adv_order) == 3) coef = IS(config_monotonic) ? 0.25 : 1.0;
      if (IS(config_thickness_adv_order) == 3 && !(A1(u, iEdge) > 0)) coef = -coef;
      A1(h_edge_tl, iEdge) = 0.5 * (A1(h_tl, cell1) + A1(h_tl, cell2)) - dc2 * (d1t + d2t) / 12. -
                             dc2 * coef * (d1t - d2t) / 12.;
      A1(h_edge, iEdge) = 0.5 * (A1(h, cell1) + A1(h, cell2)) - dc2 * (d1 + d2) / 12. -
                          dc2 * coef * (d1 - d2) / 12.;
    }
  } else {
    for (iEdge = 1; iEdge <= nEdges; iEdge++) { /* :117-126 */
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      if (cell1 <= nCells && cell2 <= nCells) {
        A1(h_edge_tl, iEdge) = 0.5 * (A1(h_tl, cell1) + A1(h_tl, cell2));
        A1(h_edge, iEdge) = 0.5 * (A1(h, cell1) + A1(h, cell2));
      }
    }
  }
  /* :255-271 */
  for (iVertex = 1; iVertex <= nVertices; iVertex++) { A1(circ_tl, iVertex) = 0.0; A1(circ, iVertex) = 0.0; }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    const int v1 = A2(verticesOnEdge, 2, 1, iEdge), v2 = A2(verticesOnEdge, 2, 2, iEdge);
    A1(circ_tl, v1) = A1(circ_tl, v1) - A1(dcEdge, iEdge) * A1(u_tl, iEdge);
    A1(circ, v1) = A1(circ, v1) - A1(dcEdge, iEdge) * A1(u, iEdge);
    A1(circ_tl, v2) = A1(circ_tl, v2) + A1(dcEdge, iEdge) * A1(u_tl, iEdge);
    A1(circ, v2) = A1(circ, v2) + A1(dcEdge, iEdge) * A1(u, iEdge);
  }
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    A1(vort_tl, iVertex) = A1(circ_tl, iVertex) / A1(areaTriangle, iVertex);
    A1(vort, iVertex) = A1(circ, iVertex) / A1(areaTriangle, iVertex);
  }
  /* :274-298 */
  for (iCell = 1; iCell <= nCells; iCell++) { A1(div_tl, iCell) = 0.0; A1(div, iCell) = 0.0; }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    if (cell1 <= nCells) {
      A1(div_tl, cell1) = A1(div_tl, cell1) + A1(u_tl, iEdge) * A1(dvEdge, iEdge);
      A1(div, cell1) = A1(div, cell1) + A1(u, iEdge) * A1(dvEdge, iEdge);
    }
    if (cell2 <= nCells) {
      A1(div_tl, cell2) = A1(div_tl, cell2) - A1(u_tl, iEdge) * A1(dvEdge, iEdge);
      A1(div, cell2) = A1(div, cell2) - A1(u, iEdge) * A1(dvEdge, iEdge);
    }
  }
  for (iCell = 1; iCell <= nCells; iCell++) {
    r = 1.0 / A1(areaCell, iCell);
    A1(div_tl, iCell) = A1(div_tl, iCell) * r;
    A1(div, iCell) = A1(div, iCell) * r;
  }
  /* :301-316 */
  for (iCell = 1; iCell <= nCells; iCell++) { A1(ke_tl, iCell) = 0.; A1(ke, iCell) = 0.0; }
  for (iCell = 1; iCell <= nCells; iCell++) {
    for (i = 1; i <= A1(nEdgesOnCell, iCell); i++) {
      iEdge = A2(edgesOnCell, maxEdges, i, iCell);
      A1(ke_tl, iCell) = A1(ke_tl, iCell) + 0.25 * A1(dcEdge, iEdge) * A1(dvEdge, iEdge) *
                                                (2. * A1(u, iEdge) * A1(u_tl, iEdge));
      A1(ke, iCell) = A1(ke, iCell) + 0.25 * A1(dcEdge, iEdge) * A1(dvEdge, iEdge) *
                                          (A1(u, iEdge) * A1(u, iEdge));
    }
    A1(ke_tl, iCell) = A1(ke_tl, iCell) / A1(areaCell, iCell);
    A1(ke, iCell) = A1(ke, iCell) / A1(areaCell, iCell);
  }
  /* :319-329 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) { A1(v_tl, iEdge) = 0.; A1(v, iEdge) = 0.0; }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    for (i = 1; i <= A1(nEdgesOnEdge, iEdge); i++) {
      eoe = A2(edgesOnEdge, maxEdges2, i, iEdge);
      A1(v_tl, iEdge) = A1(v_tl, iEdge) + A2(w, maxEdges2, i, iEdge) * A1(u_tl, eoe);
      A1(v, iEdge) = A1(v, iEdge) + A2(w, maxEdges2, i, iEdge) * A1(u, eoe);
    }
  }
  /* :344-360 */
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    A1(h_vertex_tl, iVertex) = 0.0;
    A1(h_vertex, iVertex) = 0.0;
    for (i = 1; i <= vertexDegree; i++) {
      const int c = A2(cellsOnVertex, vertexDegree, i, iVertex);
      A1(h_vertex_tl, iVertex) = A1(h_vertex_tl, iVertex) + A1(h_tl, c) * A2(kite, vertexDegree, i, iVertex);
      A1(h_vertex, iVertex) = A1(h_vertex, iVertex) + A1(h, c) * A2(kite, vertexDegree, i, iVertex);
    }
    A1(h_vertex_tl, iVertex) = A1(h_vertex_tl, iVertex) / A1(areaTriangle, iVertex);
    A1(h_vertex, iVertex) = A1(h_vertex, iVertex) / A1(areaTriangle, iVertex);
    const double hv = A1(h_vertex, iVertex);
    A1(pvv_tl, iVertex) = A1(vort_tl, iVertex) / hv -
                          A1(h_vertex_tl, iVertex) * (A1(fVertex, iVertex) + A1(vort, iVertex)) / (hv * hv);
    A1(pvv, iVertex) = (A1(fVertex, iVertex) + A1(vort, iVertex)) / hv;
  }
  /* :364-369 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    const int v1 = A2(verticesOnEdge, 2, 1, iEdge), v2 = A2(verticesOnEdge, 2, 2, iEdge);
    A1(gpt_tl, iEdge) = (A1(pvv_tl, v2) - A1(pvv_tl, v1)) / A1(dvEdge, iEdge);
    A1(gpt, iEdge) = (A1(pvv, v2) - A1(pvv, v1)) / A1(dvEdge, iEdge);
  }
  /* :373-383 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) { A1(pe_tl, iEdge) = 0.0; A1(pe, iEdge) = 0.0; }
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    for (i = 1; i <= vertexDegree; i++) {
      iEdge = A2(edgesOnVertex, vertexDegree, i, iVertex);
      A1(pe_tl, iEdge) = A1(pe_tl, iEdge) + 0.5 * A1(pvv_tl, iVertex);
      A1(pe, iEdge) = A1(pe, iEdge) + 0.5 * A1(pvv, iVertex);
    }
  }
  /* :386-393 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    A1(pe_tl, iEdge) = A1(pe_tl, iEdge) - apvm * A1(v_tl, iEdge) * dt * A1(gpt, iEdge) -
                       apvm * A1(v, iEdge) * dt * A1(gpt_tl, iEdge);
    A1(pe, iEdge) = A1(pe, iEdge) - apvm * A1(v, iEdge) * dt * A1(gpt, iEdge);
  }
  /* :397-421 */
  for (iCell = 1; iCell <= nCells; iCell++) {
    A1(pc_tl, iCell) = 0.0; A1(pc, iCell) = 0.0; A1(vc_tl, iCell) = 0.0; A1(vc, iCell) = 0.0;
  }
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    for (i = 1; i <= vertexDegree; i++) {
      iCell = A2(cellsOnVertex, vertexDegree, i, iVertex);
      if (iCell <= nCells) {
        const double k = A2(kite, vertexDegree, i, iVertex), ac = A1(areaCell, iCell);
        A1(pc_tl, iCell) = A1(pc_tl, iCell) + k * A1(pvv_tl, iVertex) / ac;
        A1(pc, iCell) = A1(pc, iCell) + k * A1(pvv, iVertex) / ac;
        A1(vc_tl, iCell) = A1(vc_tl, iCell) + k * A1(vort_tl, iVertex) / ac;
        A1(vc, iCell) = A1(vc, iCell) + k * A1(vort, iVertex) / ac;
      }
    }
  }
  /* :425-434 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) { A1(gpn_tl, iEdge) = 0.0; A1(gpn, iEdge) = 0.0; }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    if (cell1 <= nCells && cell2 <= nCells) {
      A1(gpn_tl, iEdge) = (A1(pc_tl, cell2) - A1(pc_tl, cell1)) / A1(dcEdge, iEdge);
      A1(gpn, iEdge) = (A1(pc, cell2) - A1(pc, cell1)) / A1(dcEdge, iEdge);
    }
  }
  /* :437-445 */
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    A1(pe_tl, iEdge) = A1(pe_tl, iEdge) - apvm * A1(u_tl, iEdge) * dt * A1(gpn, iEdge) -
                       apvm * A1(u, iEdge) * dt * A1(gpn_tl, iEdge);
    A1(pe, iEdge) = A1(pe, iEdge) - apvm * A1(u, iEdge) * dt * A1(gpn, iEdge);
  }
}

/* sw_compute_tend_tlm: src/mpas_sw_dyncore_tlm.f90:449-770 */
static void tend_tlm(orc_mod *m, const double *h, const double *h_tl, const double *u,
                     const double *u_tl) {
  const int nCells = IS(nCells), nEdges = IS(nEdges), nVertices = IS(nVertices);
  const int maxEdges2 = IS(maxEdges2);
  const int *cellsOnEdge = I(cellsOnEdge), *verticesOnEdge = I(verticesOnEdge);
  const int *edgesOnEdge = I(edgesOnEdge), *nEdgesOnEdge = I(nEdgesOnEdge);
  const double *dcEdge = R(dcEdge), *dvEdge = R(dvEdge), *areaCell = R(areaCell);
  const double *areaTriangle = R(areaTriangle), *h_s = R(h_s), *u_src = R(u_src);
  const double *w = R(weightsOnEdge), *sc2 = R(meshScalingDel2), *sc4 = R(meshScalingDel4);
  const double visc2 = RS(config_h_mom_eddy_visc2), visc4 = RS(config_h_mom_eddy_visc4);
  const double *he = R(h_edge), *he_tl = R(h_edge_tl), *ke = R(ke), *ke_tl = R(ke_tl);
  const double *pe = R(pv_edge), *pe_tl = R(pv_edge_tl);
  const double *div = R(divergence), *div_tl = R(divergence_tl), *vort = R(vorticity), *vort_tl = R(vorticity_tl);
  double *th = R(tend_h), *th_tl = R(tend_h_tl), *tu = R(tend_u), *tu_tl = R(tend_u_tl);
  int iEdge, iCell, iVertex, j, cell1, cell2, vertex1, vertex2, eoe;
  double flux, flux_tl, q, q_tl, workpv, workpv_tl, r, ud, ud_tl, ke_edge, ke_edge_tl;

  for (iCell = 1; iCell <= nCells; iCell++) { A1(th_tl, iCell) = 0.0; A1(th, iCell) = 0.0; }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) { /* :543-555 */
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    flux_tl = A1(u_tl, iEdge) * A1(dvEdge, iEdge) * A1(he, iEdge) +
              A1(u, iEdge) * A1(dvEdge, iEdge) * A1(he_tl, iEdge);
    flux = A1(u, iEdge) * A1(dvEdge, iEdge) * A1(he, iEdge);
    A1(th_tl, cell1) = A1(th_tl, cell1) - flux_tl;
    A1(th, cell1) = A1(th, cell1) - flux;
    A1(th_tl, cell2) = A1(th_tl, cell2) + flux_tl;
    A1(th, cell2) = A1(th, cell2) + flux;
  }
  for (iCell = 1; iCell <= nCells; iCell++) {
    A1(th_tl, iCell) = A1(th_tl, iCell) / A1(areaCell, iCell);
    A1(th, iCell) = A1(th, iCell) / A1(areaCell, iCell);
  }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) { A1(tu_tl, iEdge) = 0.0; A1(tu, iEdge) = 0.0; }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) { /* :566-595 */
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    q_tl = 0.;
    q = 0.0;
    for (j = 1; j <= A1(nEdgesOnEdge, iEdge); j++) {
      eoe = A2(edgesOnEdge, maxEdges2, j, iEdge);
      const double wj = A2(w, maxEdges2, j, iEdge);
      workpv_tl = 0.5 * (A1(pe_tl, iEdge) + A1(pe_tl, eoe));
      workpv = 0.5 * (A1(pe, iEdge) + A1(pe, eoe));
      q_tl = q_tl + wj * A1(u_tl, eoe) * workpv * A1(he, eoe) +
             wj * A1(u, eoe) * workpv_tl * A1(he, eoe) + wj * A1(u, eoe) * workpv * A1(he_tl, eoe);
      q = q + wj * A1(u, eoe) * workpv * A1(he, eoe);
    }
    A1(tu_tl, iEdge) = q_tl - (A1(ke_tl, cell2) - A1(ke_tl, cell1) +
                               GRAVITY * (A1(h_tl, cell2) - A1(h_tl, cell1))) / A1(dcEdge, iEdge);
    A1(tu, iEdge) = q - (A1(ke, cell2) - A1(ke, cell1) +
                         GRAVITY * (A1(h, cell2) + A1(h_s, cell2) - A1(h, cell1) - A1(h_s, cell1))) /
                            A1(dcEdge, iEdge);
  }
  if (visc2 > 0.0) { /* :600-618 */
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      ud_tl = (A1(div_tl, cell2) - A1(div_tl, cell1)) / A1(dcEdge, iEdge) -
              (A1(vort_tl, vertex2) - A1(vort_tl, vertex1)) / A1(dvEdge, iEdge);
      ud = (A1(div, cell2) - A1(div, cell1)) / A1(dcEdge, iEdge) -
           (A1(vort, vertex2) - A1(vort, vertex1)) / A1(dvEdge, iEdge);
      ud_tl = A1(sc2, iEdge) * visc2 * ud_tl;
      ud = A1(sc2, iEdge) * visc2 * ud;
      A1(tu_tl, iEdge) = A1(tu_tl, iEdge) + ud_tl;
      A1(tu, iEdge) = A1(tu, iEdge) + ud;
    }
  }
  if (visc4 > 0.0) { /* :624-740 */
    double *dd_tl = dalloc(nCells + 1), *dd = dalloc(nCells + 1), *du_tl = dalloc(nEdges + 1),
           *du = dalloc(nEdges + 1), *dc_tl = dalloc(nVertices + 1), *dcirc = dalloc(nVertices + 1),
           *dv_tl = dalloc(nVertices + 1), *dvort = dalloc(nVertices + 1);
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      A1(du_tl, iEdge) = (A1(div_tl, cell2) - A1(div_tl, cell1)) / A1(dcEdge, iEdge) -
                         (A1(vort_tl, vertex2) - A1(vort_tl, vertex1)) / A1(dvEdge, iEdge);
      A1(du, iEdge) = (A1(div, cell2) - A1(div, cell1)) / A1(dcEdge, iEdge) -
                      (A1(vort, vertex2) - A1(vort, vertex1)) / A1(dvEdge, iEdge);
    }
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      A1(dc_tl, vertex1) = A1(dc_tl, vertex1) - A1(dcEdge, iEdge) * A1(du_tl, iEdge);
      A1(dcirc, vertex1) = A1(dcirc, vertex1) - A1(dcEdge, iEdge) * A1(du, iEdge);
      A1(dc_tl, vertex2) = A1(dc_tl, vertex2) + A1(dcEdge, iEdge) * A1(du_tl, iEdge);
      A1(dcirc, vertex2) = A1(dcirc, vertex2) + A1(dcEdge, iEdge) * A1(du, iEdge);
    }
    for (iVertex = 1; iVertex <= nVertices; iVertex++) {
      r = 1.0 / A1(areaTriangle, iVertex);
      A1(dv_tl, iVertex) = A1(dc_tl, iVertex) * r;
      A1(dvort, iVertex) = A1(dcirc, iVertex) * r;
    }
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      A1(dd_tl, cell1) = A1(dd_tl, cell1) + A1(du_tl, iEdge) * A1(dvEdge, iEdge);
      A1(dd, cell1) = A1(dd, cell1) + A1(du, iEdge) * A1(dvEdge, iEdge);
      A1(dd_tl, cell2) = A1(dd_tl, cell2) - A1(du_tl, iEdge) * A1(dvEdge, iEdge);
      A1(dd, cell2) = A1(dd, cell2) - A1(du, iEdge) * A1(dvEdge, iEdge);
    }
    for (iCell = 1; iCell <= nCells; iCell++) {
      r = 1.0 / A1(areaCell, iCell);
      A1(dd_tl, iCell) = A1(dd_tl, iCell) * r;
      A1(dd, iCell) = A1(dd, iCell) * r;
    }
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      ud_tl = (A1(dd_tl, cell2) - A1(dd_tl, cell1)) / A1(dcEdge, iEdge) -
              (A1(dv_tl, vertex2) - A1(dv_tl, vertex1)) / A1(dvEdge, iEdge);
      ud = (A1(dd, cell2) - A1(dd, cell1)) / A1(dcEdge, iEdge) -
           (A1(dvort, vertex2) - A1(dvort, vertex1)) / A1(dvEdge, iEdge);
      ud_tl = A1(sc4, iEdge) * visc4 * ud_tl;
      ud = A1(sc4, iEdge) * visc4 * ud;
      A1(tu_tl, iEdge) = A1(tu_tl, iEdge) - ud_tl;
      A1(tu, iEdge) = A1(tu, iEdge) - ud;
    }
    free(dd_tl); free(dd); free(du_tl); free(du); free(dc_tl); free(dcirc); free(dv_tl); free(dvort);
  }
  if (IS(config_wind_stress)) { /* :743-750 */
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      const double hh = A1(he, iEdge);
      A1(tu_tl, iEdge) = A1(tu_tl, iEdge) - A1(he_tl, iEdge) * A1(u_src, iEdge) / RHO_REF / (hh * hh);
      A1(tu, iEdge) = A1(tu, iEdge) + A1(u_src, iEdge) / RHO_REF / hh;
    }
  }
  if (IS(config_bottom_drag)) { /* :752-768 */
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      ke_edge_tl = 0.5 * (A1(ke_tl, cell1) + A1(ke_tl, cell2));
      ke_edge = 0.5 * (A1(ke, cell1) + A1(ke, cell2));
      const double hh = A1(he, iEdge), uu = A1(u, iEdge);
      A1(tu_tl, iEdge) = A1(tu_tl, iEdge) - 1.0e-3 * A1(u_tl, iEdge) * sqrt(2.0 * ke_edge) / hh -
                         0.5 * 1.0e-3 * uu * (2.0 * ke_edge_tl) / sqrt(2.0 * ke_edge) / hh +
                         1.0e-3 * uu * sqrt(2.0 * ke_edge) * A1(he_tl, iEdge) / (hh * hh);
      A1(tu, iEdge) = A1(tu, iEdge) - 1.0e-3 * uu * sqrt(2.0 * ke_edge) / hh;
    }
  }
}

/* mpas_reconstruct_2d_tlm: src/mpas_sw_dyncore_tlm.f90:772-870 */
static void reconstruct_tlm(orc_mod *m, const double *u, const double *u_tl) {
  const int nCells = IS(nCells), maxEdges = IS(maxEdges);
  const double *cr = R(coeffs_reconstruct);
  double *X = R(uReconstructX), *Y = R(uReconstructY), *Z = R(uReconstructZ);
  double *Xt = R(uReconstructX_tl), *Yt = R(uReconstructY_tl), *Zt = R(uReconstructZ_tl);
  for (int c = 1; c <= nCells; c++) {
    A1(Xt, c) = 0.0; A1(X, c) = 0.0; A1(Yt, c) = 0.0; A1(Y, c) = 0.0; A1(Zt, c) = 0.0; A1(Z, c) = 0.0;
    for (int i = 1; i <= A1(I(nEdgesOnCell), c); i++) {
      const int e = A2(I(edgesOnCell), maxEdges, i, c);
      A1(Xt, c) = A1(Xt, c) + A3(cr, 3, maxEdges, 1, i, c) * A1(u_tl, e);
      A1(X, c) = A1(X, c) + A3(cr, 3, maxEdges, 1, i, c) * A1(u, e);
      A1(Yt, c) = A1(Yt, c) + A3(cr, 3, maxEdges, 2, i, c) * A1(u_tl, e);
      A1(Y, c) = A1(Y, c) + A3(cr, 3, maxEdges, 2, i, c) * A1(u, e);
      A1(Zt, c) = A1(Zt, c) + A3(cr, 3, maxEdges, 3, i, c) * A1(u_tl, e);
      A1(Z, c) = A1(Z, c) + A3(cr, 3, maxEdges, 3, i, c) * A1(u, e);
    }
  }
  double *Zo = R(uReconstructZonal), *Zot = R(uReconstructZonal_tl);
  double *Me = R(uReconstructMeridional), *Met = R(uReconstructMeridional_tl);
  for (int c = 1; c <= nCells; c++) {
    if (IS(on_a_sphere)) {
      const double clat = cos(A1(R(latCell), c)), slat = sin(A1(R(latCell), c));
      const double clon = cos(A1(R(lonCell), c)), slon = sin(A1(R(lonCell), c));
      A1(Zot, c) = -A1(Xt, c) * slon + A1(Yt, c) * clon;
      A1(Zo, c) = -A1(X, c) * slon + A1(Y, c) * clon;
      A1(Met, c) = -(A1(Xt, c) * clon + A1(Yt, c) * slon) * slat + A1(Zt, c) * clat;
      A1(Me, c) = -(A1(X, c) * clon + A1(Y, c) * slon) * slat + A1(Z, c) * clat;
    } else {
      A1(Zot, c) = A1(Xt, c); A1(Zo, c) = A1(X, c); A1(Met, c) = A1(Yt, c); A1(Me, c) = A1(Y, c);
    }
  }
}

/* ---------------------------------------------------------------------------------------- */
/* Adjoint: src/mpas_sw_dyncore_adj.f90                                                       */
/* ---------------------------------------------------------------------------------------- */
/* sw_compute_solve_diagnostics_adj :1-453 (order 2; orders 3/4 restated at the end) */
static void diag_adj(orc_mod *m, double dt, const double *h, double *h_ad, const double *u,
                     double *u_ad) {
  const int nCells = IS(nCells), nEdges = IS(nEdges), nVertices = IS(nVertices);
  const int maxEdges = IS(maxEdges), maxEdges2 = IS(maxEdges2), vertexDegree = IS(vertexDegree);
  const int *cellsOnEdge = I(cellsOnEdge), *verticesOnEdge = I(verticesOnEdge);
  const int *edgesOnCell = I(edgesOnCell), *edgesOnEdge = I(edgesOnEdge);
  const int *edgesOnVertex = I(edgesOnVertex), *cellsOnVertex = I(cellsOnVertex);
  const int *nEdgesOnCell = I(nEdgesOnCell), *nEdgesOnEdge = I(nEdgesOnEdge);
  const double *dcEdge = R(dcEdge), *dvEdge = R(dvEdge), *areaCell = R(areaCell);
  const double *areaTriangle = R(areaTriangle), *fVertex = R(fVertex);
  const double *w = R(weightsOnEdge), *kite = R(kiteAreasOnVertex);
  const double apvm = RS(config_apvm_upwinding);
  double *v_ad = R(v_ad), *he_ad = R(h_edge_ad), *hv_ad = R(h_vertex_ad), *pe_ad = R(pv_edge_ad);
  double *pvv_ad = R(pv_vertex_ad), *pc_ad = R(pv_cell_ad), *circ_ad = R(circulation_ad);
  double *vort_ad = R(vorticity_ad), *div_ad = R(divergence_ad), *ke_ad = R(ke_ad);
  double *vc_ad = R(vorticity_cell_ad), *gpn_ad = R(gradPVn_ad), *gpt_ad = R(gradPVt_ad);
  /* local forward recomputation :127-188 */
  double *circ = dalloc(nVertices), *vort = dalloc(nVertices), *v = dalloc(nEdges);
  double *hv = dalloc(nVertices), *pvv = dalloc(nVertices), *gpt = dalloc(nEdges);
  double *pc = dalloc(nCells), *gpn = dalloc(nEdges);
  int iEdge, iCell, iVertex, i, cell1, cell2, eoe;
  double r;

  for (iCell = 1; iCell <= nCells; iCell++) A1(I(boundaryCell), iCell) = 0;

  for (iVertex = 1; iVertex <= nVertices; iVertex++) A1(circ, iVertex) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    const int v1 = A2(verticesOnEdge, 2, 1, iEdge), v2 = A2(verticesOnEdge, 2, 2, iEdge);
    A1(circ, v1) = A1(circ, v1) - A1(dcEdge, iEdge) * A1(u, iEdge);
    A1(circ, v2) = A1(circ, v2) + A1(dcEdge, iEdge) * A1(u, iEdge);
  }
  for (iVertex = 1; iVertex <= nVertices; iVertex++)
    A1(vort, iVertex) = A1(circ, iVertex) / A1(areaTriangle, iVertex);
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(v, iEdge) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++)
    for (i = 1; i <= A1(nEdgesOnEdge, iEdge); i++) {
      eoe = A2(edgesOnEdge, maxEdges2, i, iEdge);
      A1(v, iEdge) = A1(v, iEdge) + A2(w, maxEdges2, i, iEdge) * A1(u, eoe);
    }
  for (iVertex = 1; iVertex <= nVertices; iVertex++) {
    A1(hv, iVertex) = 0.0;
    for (i = 1; i <= vertexDegree; i++)
      A1(hv, iVertex) = A1(hv, iVertex) + A1(h, A2(cellsOnVertex, vertexDegree, i, iVertex)) *
                                              A2(kite, vertexDegree, i, iVertex);
    A1(hv, iVertex) = A1(hv, iVertex) / A1(areaTriangle, iVertex);
    A1(pvv, iVertex) = (A1(fVertex, iVertex) + A1(vort, iVertex)) / A1(hv, iVertex);
  }
  for (iEdge = 1; iEdge <= nEdges; iEdge++)
    A1(gpt, iEdge) = (A1(pvv, A2(verticesOnEdge, 2, 2, iEdge)) - A1(pvv, A2(verticesOnEdge, 2, 1, iEdge))) /
                     A1(dvEdge, iEdge);
  for (iCell = 1; iCell <= nCells; iCell++) A1(pc, iCell) = 0.0;
  for (iVertex = 1; iVertex <= nVertices; iVertex++)
    for (i = 1; i <= vertexDegree; i++) {
      iCell = A2(cellsOnVertex, vertexDegree, i, iVertex);
      if (iCell <= nCells)
        A1(pc, iCell) = A1(pc, iCell) + A2(kite, vertexDegree, i, iVertex) * A1(pvv, iVertex) / A1(areaCell, iCell);
    }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(gpn, iEdge) = 0.0;
  for (iEdge = 1; iEdge <= nEdges; iEdge++)
    if (A2(cellsOnEdge, 2, 1, iEdge) <= nCells && A2(cellsOnEdge, 2, 2, iEdge) <= nCells)
      A1(gpn, iEdge) = (A1(pc, A2(cellsOnEdge, 2, 2, iEdge)) - A1(pc, A2(cellsOnEdge, 2, 1, iEdge))) /
                       A1(dcEdge, iEdge);

  /* :193-200 */
  for (iEdge = nEdges; iEdge >= 1; iEdge--) {
    A1(gpn_ad, iEdge) = A1(gpn_ad, iEdge) - apvm * A1(u, iEdge) * dt * A1(pe_ad, iEdge);
    A1(u_ad, iEdge) = A1(u_ad, iEdge) - apvm * dt * A1(gpn, iEdge) * A1(pe_ad, iEdge);
  }
  /* :202-213 */
  for (iEdge = nEdges; iEdge >= 1; iEdge--) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    if (cell1 <= nCells && cell2 <= nCells) {
      A1(pc_ad, cell1) = A1(pc_ad, cell1) - A1(gpn_ad, iEdge) / A1(dcEdge, iEdge);
      A1(pc_ad, cell2) = A1(pc_ad, cell2) + A1(gpn_ad, iEdge) / A1(dcEdge, iEdge);
      A1(gpn_ad, iEdge) = 0.;
    }
  }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(gpn_ad, iEdge) = 0.0;
  /* :215-229 */
  for (iVertex = nVertices; iVertex >= 1; iVertex--)
    for (i = vertexDegree; i >= 1; i--) {
      iCell = A2(cellsOnVertex, vertexDegree, i, iVertex);
      if (iCell <= nCells) {
        const double k = A2(kite, vertexDegree, i, iVertex);
        A1(vort_ad, iVertex) = A1(vort_ad, iVertex) + k / A1(areaCell, iCell) * A1(vc_ad, iCell);
        A1(pvv_ad, iVertex) = A1(pvv_ad, iVertex) + k / A1(areaCell, iCell) * A1(pc_ad, iCell);
      }
    }
  for (iCell = 1; iCell <= nCells; iCell++) { A1(vc_ad, iCell) = 0.0; A1(pc_ad, iCell) = 0.0; }
  /* :235-242 */
  for (iEdge = nEdges; iEdge >= 1; iEdge--) {
    A1(gpt_ad, iEdge) = A1(gpt_ad, iEdge) - apvm * A1(v, iEdge) * dt * A1(pe_ad, iEdge);
    A1(v_ad, iEdge) = A1(v_ad, iEdge) - apvm * dt * A1(gpt, iEdge) * A1(pe_ad, iEdge);
  }
  /* :244-252 */
  for (iVertex = nVertices; iVertex >= 1; iVertex--)
    for (i = vertexDegree; i >= 1; i--) {
      iEdge = A2(edgesOnVertex, vertexDegree, i, iVertex);
      A1(pvv_ad, iVertex) = A1(pvv_ad, iVertex) + 0.5 * A1(pe_ad, iEdge);
    }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(pe_ad, iEdge) = 0.0;
  /* :254-262 */
  for (iEdge = nEdges; iEdge >= 1; iEdge--) {
    const int v1 = A2(verticesOnEdge, 2, 1, iEdge), v2 = A2(verticesOnEdge, 2, 2, iEdge);
    A1(pvv_ad, v1) = A1(pvv_ad, v1) - A1(gpt_ad, iEdge) / A1(dvEdge, iEdge);
    A1(pvv_ad, v2) = A1(pvv_ad, v2) + A1(gpt_ad, iEdge) / A1(dvEdge, iEdge);
    A1(gpt_ad, iEdge) = 0.;
  }
  /* :268-292 */
  for (iVertex = nVertices; iVertex >= 1; iVertex--) {
    const double hh = A1(hv, iVertex);
    A1(hv_ad, iVertex) = A1(hv_ad, iVertex) -
                         (A1(fVertex, iVertex) + A1(vort, iVertex)) / (hh * hh) * A1(pvv_ad, iVertex);
    A1(vort_ad, iVertex) = A1(vort_ad, iVertex) + A1(pvv_ad, iVertex) / hh;
    A1(pvv_ad, iVertex) = 0.;
    A1(hv_ad, iVertex) = A1(hv_ad, iVertex) / A1(areaTriangle, iVertex);
    for (i = vertexDegree; i >= 1; i--) {
      const int c = A2(cellsOnVertex, vertexDegree, i, iVertex);
      A1(h_ad, c) = A1(h_ad, c) + A2(kite, vertexDegree, i, iVertex) * A1(hv_ad, iVertex);
    }
    A1(hv_ad, iVertex) = 0.0;
  }
  /* :296-304 */
  for (iEdge = nEdges; iEdge >= 1; iEdge--)
    for (i = A1(nEdgesOnEdge, iEdge); i >= 1; i--) {
      eoe = A2(edgesOnEdge, maxEdges2, i, iEdge);
      A1(u_ad, eoe) = A1(u_ad, eoe) + A2(w, maxEdges2, i, iEdge) * A1(v_ad, iEdge);
    }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(v_ad, iEdge) = 0.;
  /* :306-318 */
  for (iCell = nCells; iCell >= 1; iCell--) {
    A1(ke_ad, iCell) = A1(ke_ad, iCell) / A1(areaCell, iCell);
    for (i = A1(nEdgesOnCell, iCell); i >= 1; i--) {
      iEdge = A2(edgesOnCell, maxEdges, i, iCell);
      A1(u_ad, iEdge) = A1(u_ad, iEdge) + 0.25 * A1(dcEdge, iEdge) * A1(dvEdge, iEdge) * 2. *
                                              A1(u, iEdge) * A1(ke_ad, iCell);
    }
  }
  for (iCell = 1; iCell <= nCells; iCell++) A1(ke_ad, iCell) = 0.;
  /* :321-341 */
  for (iCell = nCells; iCell >= 1; iCell--) {
    r = 1.0 / A1(areaCell, iCell);
    A1(div_ad, iCell) = A1(div_ad, iCell) * r;
  }
  for (iEdge = nEdges; iEdge >= 1; iEdge--) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    if (cell2 <= nCells) A1(u_ad, iEdge) = A1(u_ad, iEdge) - A1(dvEdge, iEdge) * A1(div_ad, cell2);
    if (cell1 <= nCells) A1(u_ad, iEdge) = A1(u_ad, iEdge) + A1(dvEdge, iEdge) * A1(div_ad, cell1);
  }
  for (iCell = 1; iCell <= nCells; iCell++) A1(div_ad, iCell) = 0.0;
  /* :343-356 */
  for (iVertex = nVertices; iVertex >= 1; iVertex--) {
    A1(circ_ad, iVertex) = A1(circ_ad, iVertex) + A1(vort_ad, iVertex) / A1(areaTriangle, iVertex);
    A1(vort_ad, iVertex) = 0.;
  }
  for (iEdge = nEdges; iEdge >= 1; iEdge--) {
    A1(u_ad, iEdge) = A1(u_ad, iEdge) + A1(dcEdge, iEdge) * A1(circ_ad, A2(verticesOnEdge, 2, 2, iEdge));
    A1(u_ad, iEdge) = A1(u_ad, iEdge) - A1(dcEdge, iEdge) * A1(circ_ad, A2(verticesOnEdge, 2, 1, iEdge));
  }
  for (iVertex = 1; iVertex <= nVertices; iVertex++) A1(circ_ad, iVertex) = 0.0;
  /* :358-451 */
  if (IS(config_thickness_adv_order) == 2) {
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      if (cell1 <= nCells && cell2 <= nCells) {
        A1(h_ad, cell2) = A1(h_ad, cell2) + 0.5 * A1(he_ad, iEdge);
        A1(h_ad, cell1) = A1(h_ad, cell1) + 0.5 * A1(he_ad, iEdge);
        A1(he_ad, iEdge) = 0.;
      }
    }
  } else {
    const double *dtw = R(deriv_two);
    double coef = 0.;
    if (IS(config_thickness_adv_order) == 3) coef = IS(config_monotonic) ? 0.25 : 1.0;
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      if (cell1 <= nCells && cell2 <= nCells) {
        const double dc2 = A1(dcEdge, iEdge) * A1(dcEdge, iEdge);
        double d2_ad, d1_ad;
        if (IS(config_thickness_adv_order) == 3) {
          if (A1(u, iEdge) > 0) {
            d2_ad = dc2 * coef / 12. * A1(he_ad, iEdge);
            d1_ad = -dc2 * coef / 12. * A1(he_ad, iEdge);
          } else {
            d2_ad = -dc2 * coef / 12. * A1(he_ad, iEdge);
            d1_ad = dc2 * coef / 12. * A1(he_ad, iEdge);
          }
          d2_ad = d2_ad - dc2 / 12. * A1(he_ad, iEdge);
          d1_ad = d1_ad - dc2 / 12. * A1(he_ad, iEdge);
        } else {
          d2_ad = -dc2 / 12. * A1(he_ad, iEdge);
          d1_ad = -dc2 / 12. * A1(he_ad, iEdge);
        }
        A1(h_ad, cell2) = A1(h_ad, cell2) + 0.5 * A1(he_ad, iEdge);
        A1(h_ad, cell1) = A1(h_ad, cell1) + 0.5 * A1(he_ad, iEdge);
        A1(he_ad, iEdge) = 0.;
        if (A1(I(boundaryCell), cell1) == 0 && A1(I(boundaryCell), cell2) == 0) {
          for (i = A1(nEdgesOnCell, cell2); i >= 1; i--) {
            const int cc = A2(I(cellsOnCell), maxEdges, i, cell2);
            A1(h_ad, cc) = A1(h_ad, cc) + A3(dtw, 15, 2, i + 1, 2, iEdge) * d2_ad;
          }
          for (i = A1(nEdgesOnCell, cell1); i >= 1; i--) {
            const int cc = A2(I(cellsOnCell), maxEdges, i, cell1);
            A1(h_ad, cc) = A1(h_ad, cc) + A3(dtw, 15, 2, i + 1, 1, iEdge) * d1_ad;
          }
          A1(h_ad, cell2) = A1(h_ad, cell2) + A3(dtw, 15, 2, 1, 2, iEdge) * d2_ad;
          A1(h_ad, cell1) = A1(h_ad, cell1) + A3(dtw, 15, 2, 1, 1, iEdge) * d1_ad;
        }
      }
    }
  }
  (void)edgesOnCell;
  free(circ); free(vort); free(v); free(hv); free(pvv); free(gpt); free(pc); free(gpn);
}

/* sw_compute_tend_adj: src/mpas_sw_dyncore_adj.f90:455-738 */
static void tend_adj(orc_mod *m, const double *h, double *h_ad, const double *u, double *u_ad) {
  const int nCells = IS(nCells), nEdges = IS(nEdges), nVertices = IS(nVertices);
  const int maxEdges2 = IS(maxEdges2);
  const int *cellsOnEdge = I(cellsOnEdge), *verticesOnEdge = I(verticesOnEdge);
  const int *edgesOnEdge = I(edgesOnEdge), *nEdgesOnEdge = I(nEdgesOnEdge);
  const double *dcEdge = R(dcEdge), *dvEdge = R(dvEdge), *areaCell = R(areaCell);
  const double *areaTriangle = R(areaTriangle), *u_src = R(u_src);
  const double *w = R(weightsOnEdge), *sc2 = R(meshScalingDel2), *sc4 = R(meshScalingDel4);
  const double visc2 = RS(config_h_mom_eddy_visc2), visc4 = RS(config_h_mom_eddy_visc4);
  const double *he = R(h_edge), *ke = R(ke), *pe = R(pv_edge);
  double *he_ad = R(h_edge_ad), *ke_ad = R(ke_ad), *pe_ad = R(pv_edge_ad);
  double *div_ad = R(divergence_ad), *vort_ad = R(vorticity_ad);
  double *tu_ad = R(tend_u_ad), *th_ad = R(tend_h_ad);
  int iEdge, iCell, iVertex, j, cell1, cell2, vertex1, vertex2, eoe;
  double ke_edge, ke_edge_ad, ud_ad, q_ad, workpv, workpv_ad, flux_ad, r;
  (void)h;

  if (IS(config_bottom_drag)) { /* :549-565 */
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      ke_edge = 0.5 * (A1(ke, cell1) + A1(ke, cell2));
      const double hh = A1(he, iEdge);
      A1(he_ad, iEdge) = A1(he_ad, iEdge) +
                         1.0e-3 * A1(u, iEdge) * sqrt(2.0 * ke_edge) / (hh * hh) * A1(tu_ad, iEdge);
      ke_edge_ad = -(0.5 * 1.0e-3 * A1(u, iEdge) * 2.0 / sqrt(2.0 * ke_edge) / hh * A1(tu_ad, iEdge));
      A1(u_ad, iEdge) = A1(u_ad, iEdge) - 1.0e-3 * sqrt(2.0 * ke_edge) / hh * A1(tu_ad, iEdge);
      A1(ke_ad, cell2) = A1(ke_ad, cell2) + 0.5 * ke_edge_ad;
      A1(ke_ad, cell1) = A1(ke_ad, cell1) + 0.5 * ke_edge_ad;
    }
  }
  if (IS(config_wind_stress)) { /* :567-572 */
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      const double hh = A1(he, iEdge);
      A1(he_ad, iEdge) = A1(he_ad, iEdge) - A1(u_src, iEdge) / RHO_REF / (hh * hh) * A1(tu_ad, iEdge);
    }
  }
  if (visc4 > 0.0) { /* :574-669 */
    double *dd_ad = dalloc(nCells + 1), *du_ad = dalloc(nEdges + 1);
    double *dc_ad = dalloc(nVertices + 1), *dv_ad = dalloc(nVertices + 1);
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      ud_ad = -A1(tu_ad, iEdge);
      ud_ad = A1(sc4, iEdge) * visc4 * ud_ad;
      A1(dv_ad, vertex1) = A1(dv_ad, vertex1) + ud_ad / A1(dvEdge, iEdge);
      A1(dv_ad, vertex2) = A1(dv_ad, vertex2) - ud_ad / A1(dvEdge, iEdge);
      A1(dd_ad, cell1) = A1(dd_ad, cell1) - ud_ad / A1(dcEdge, iEdge);
      A1(dd_ad, cell2) = A1(dd_ad, cell2) + ud_ad / A1(dcEdge, iEdge);
    }
    for (iCell = nCells; iCell >= 1; iCell--) {
      r = 1.0 / A1(areaCell, iCell);
      A1(dd_ad, iCell) = A1(dd_ad, iCell) * r;
    }
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      A1(du_ad, iEdge) = A1(du_ad, iEdge) - A1(dvEdge, iEdge) * A1(dd_ad, cell2);
      A1(du_ad, iEdge) = A1(du_ad, iEdge) + A1(dvEdge, iEdge) * A1(dd_ad, cell1);
    }
    for (iVertex = nVertices; iVertex >= 1; iVertex--) {
      r = 1.0 / A1(areaTriangle, iVertex);
      A1(dc_ad, iVertex) = A1(dc_ad, iVertex) + A1(dv_ad, iVertex) * r;
      A1(dv_ad, iVertex) = 0.;
    }
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      A1(du_ad, iEdge) = A1(du_ad, iEdge) + A1(dcEdge, iEdge) * A1(dc_ad, vertex2);
      A1(du_ad, iEdge) = A1(du_ad, iEdge) - A1(dcEdge, iEdge) * A1(dc_ad, vertex1);
    }
    for (iEdge = nEdges; iEdge >= 1; iEdge--) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      A1(vort_ad, vertex1) = A1(vort_ad, vertex1) + A1(du_ad, iEdge) / A1(dvEdge, iEdge);
      A1(vort_ad, vertex2) = A1(vort_ad, vertex2) - A1(du_ad, iEdge) / A1(dvEdge, iEdge);
      A1(div_ad, cell1) = A1(div_ad, cell1) - A1(du_ad, iEdge) / A1(dcEdge, iEdge);
      A1(div_ad, cell2) = A1(div_ad, cell2) + A1(du_ad, iEdge) / A1(dcEdge, iEdge);
    }
    free(dd_ad); free(du_ad); free(dc_ad); free(dv_ad);
  }
  if (visc2 > 0.0) { /* :671-687 (forward edge order in the reference) */
    for (iEdge = 1; iEdge <= nEdges; iEdge++) {
      cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
      vertex1 = A2(verticesOnEdge, 2, 1, iEdge); vertex2 = A2(verticesOnEdge, 2, 2, iEdge);
      ud_ad = A1(tu_ad, iEdge);
      ud_ad = A1(sc2, iEdge) * visc2 * ud_ad;
      A1(vort_ad, vertex1) = A1(vort_ad, vertex1) + ud_ad / A1(dvEdge, iEdge);
      A1(vort_ad, vertex2) = A1(vort_ad, vertex2) - ud_ad / A1(dvEdge, iEdge);
      A1(div_ad, cell1) = A1(div_ad, cell1) - ud_ad / A1(dcEdge, iEdge);
      A1(div_ad, cell2) = A1(div_ad, cell2) + ud_ad / A1(dcEdge, iEdge);
    }
  }
  /* :689-718 */
  for (iEdge = nEdges; iEdge >= 1; iEdge--) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    const double t = A1(tu_ad, iEdge), dce = A1(dcEdge, iEdge);
    A1(h_ad, cell1) = A1(h_ad, cell1) + GRAVITY / dce * t;
    A1(h_ad, cell2) = A1(h_ad, cell2) - GRAVITY / dce * t;
    A1(ke_ad, cell1) = A1(ke_ad, cell1) + t / dce;
    A1(ke_ad, cell2) = A1(ke_ad, cell2) - t / dce;
    q_ad = t;
    A1(tu_ad, iEdge) = 0.;
    for (j = A1(nEdgesOnEdge, iEdge); j >= 1; j--) {
      eoe = A2(edgesOnEdge, maxEdges2, j, iEdge);
      const double wj = A2(w, maxEdges2, j, iEdge);
      workpv = 0.5 * (A1(pe, iEdge) + A1(pe, eoe));
      A1(he_ad, eoe) = A1(he_ad, eoe) + wj * A1(u, eoe) * workpv * q_ad;
      workpv_ad = wj * A1(u, eoe) * A1(he, eoe) * q_ad;
      A1(u_ad, eoe) = A1(u_ad, eoe) + wj * workpv * A1(he, eoe) * q_ad;
      A1(pe_ad, eoe) = A1(pe_ad, eoe) + 0.5 * workpv_ad;
      A1(pe_ad, iEdge) = A1(pe_ad, iEdge) + 0.5 * workpv_ad;
    }
  }
  for (iEdge = 1; iEdge <= nEdges; iEdge++) A1(tu_ad, iEdge) = 0.0;
  /* :720-736 */
  for (iCell = nCells; iCell >= 1; iCell--) A1(th_ad, iCell) = A1(th_ad, iCell) / A1(areaCell, iCell);
  for (iEdge = 1; iEdge <= nEdges; iEdge++) {
    cell1 = A2(cellsOnEdge, 2, 1, iEdge); cell2 = A2(cellsOnEdge, 2, 2, iEdge);
    flux_ad = A1(th_ad, cell2);
    flux_ad = flux_ad - A1(th_ad, cell1);
    A1(he_ad, iEdge) = A1(he_ad, iEdge) + A1(u, iEdge) * A1(dvEdge, iEdge) * flux_ad;
    A1(u_ad, iEdge) = A1(u_ad, iEdge) + A1(dvEdge, iEdge) * A1(he, iEdge) * flux_ad;
  }
  for (iCell = 1; iCell <= nCells; iCell++) A1(th_ad, iCell) = 0.0;
}

/* mpas_reconstruct_2d_adj: src/mpas_sw_dyncore_adj.f90:740-831 */
static void reconstruct_adj(orc_mod *m, double *u_ad) {
  const int nCells = IS(nCells), maxEdges = IS(maxEdges);
  const double *cr = R(coeffs_reconstruct);
  double *Xa = R(uReconstructX_ad), *Ya = R(uReconstructY_ad), *Za = R(uReconstructZ_ad);
  double *Zoa = R(uReconstructZonal_ad), *Mea = R(uReconstructMeridional_ad);
  if (IS(on_a_sphere)) {
    for (int c = nCells; c >= 1; c--) {
      const double clat = cos(A1(R(latCell), c)), slat = sin(A1(R(latCell), c));
      const double clon = cos(A1(R(lonCell), c)), slon = sin(A1(R(lonCell), c));
      A1(Za, c) = A1(Za, c) + clat * A1(Mea, c);
      A1(Ya, c) = A1(Ya, c) - slon * slat * A1(Mea, c);
      A1(Xa, c) = A1(Xa, c) - clon * slat * A1(Mea, c);
      A1(Mea, c) = 0.0;
      A1(Ya, c) = A1(Ya, c) + clon * A1(Zoa, c);
      A1(Xa, c) = A1(Xa, c) - slon * A1(Zoa, c);
      A1(Zoa, c) = 0.0;
    }
  } else {
    for (int c = nCells; c >= 1; c--) {
      A1(Ya, c) = A1(Ya, c) + A1(Mea, c); A1(Mea, c) = 0.0;
      A1(Xa, c) = A1(Xa, c) + A1(Zoa, c); A1(Zoa, c) = 0.0;
    }
  }
  for (int c = nCells; c >= 1; c--) {
    for (int i = A1(I(nEdgesOnCell), c); i >= 1; i--) {
      const int e = A2(I(edgesOnCell), maxEdges, i, c);
      A1(u_ad, e) = A1(u_ad, e) + A3(cr, 3, maxEdges, 3, i, c) * A1(Za, c);
      A1(u_ad, e) = A1(u_ad, e) + A3(cr, 3, maxEdges, 2, i, c) * A1(Ya, c);
      A1(u_ad, e) = A1(u_ad, e) + A3(cr, 3, maxEdges, 1, i, c) * A1(Xa, c);
    }
    A1(Xa, c) = 0.0; A1(Ya, c) = 0.0; A1(Za, c) = 0.0;
  }
}

/* ---------------------------------------------------------------------------------------- */
/* Module drivers: src/mpas_sw_module.f90:495-1218                                            */
/* ---------------------------------------------------------------------------------------- */
static int check(orc_mod *m) {
  if (IS(nVertLevels) != 1) { fprintf(stderr, "oracle: nVertLevels must be 1\n"); return 1; }
  return 0;
}

/* level extraction of x(2,1,n) (the f2py/gfortran copy-in of the section x(t,:,:)) */
static void get_level(const double *x2, int n, int t, double *dst) {
  for (int i = 1; i <= n; i++) A1(dst, i) = A2(x2, 2, t, i);
}
static void put_level(double *x2, int n, int t, const double *src) {
  for (int i = 1; i <= n; i++) A2(x2, 2, t, i) = A1(src, i);
}

#define DIAG_FWD(h_, u_)                                                                      \
  diag_fwd(m, dt, h_, u_, R(v), R(h_edge), R(h_vertex), R(circulation), R(vorticity),          \
           R(divergence), R(ke), R(pv_edge), R(pv_vertex), R(pv_cell), R(vorticity_cell),     \
           R(gradPVn), R(gradPVt))
#define TEND_FWD(h_, u_) \
  tend_fwd(m, h_, u_, R(h_edge), R(vorticity), R(divergence), R(ke), R(pv_edge), R(tend_h), R(tend_u))
#define RECON(u_)                                                                       \
  reconstruct_fwd(m, u_, R(uReconstructX), R(uReconstructY), R(uReconstructZ), \
                  R(uReconstructZonal), R(uReconstructMeridional))

int orc_sw_mpas_init_block(orc_mod *m) { /* :495-526 */
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  const double dt = RS(config_dt);
  double *h1 = dalloc(nC), *u1 = dalloc(nE);
  get_level(R(h), nC, 1, h1);
  get_level(R(u), nE, 1, u1);
  DIAG_FWD(h1, u1);
  mesh_scaling(m);
  initialize_vectors(m);
  init_reconstruct(m);
  RECON(u1);
  free(h1); free(u1);
  return 0;
}

int orc_sw_rk4(orc_mod *m) { /* :528-635 */
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges), nT = IS(nTracers);
  const double dt = RS(config_dt);
  double rk_weights[4], rk_substep_weights[4];
  double *uP = dalloc(nE), *hP = dalloc(nC), *u1 = dalloc(nE), *h1 = dalloc(nC), *u2 = dalloc(nE),
         *h2 = dalloc(nC);
  double *tu = R(tend_u), *th = R(tend_h);
  get_level(R(h), nC, 1, h1);
  get_level(R(u), nE, 1, u1);
  DIAG_FWD(h1, u1);
  RECON(u1);
  memcpy(uP, u1, sizeof(double) * nE);
  memcpy(hP, h1, sizeof(double) * nC);
  memcpy(u2, u1, sizeof(double) * nE);
  memcpy(h2, h1, sizeof(double) * nC);
  for (int i = 0; i < nT * nC; i++) A2(R(tracers), 2, 2, i + 1) = A2(R(tracers), 2, 1, i + 1);
  /* tracer transport (opt-in, MPAS's mass-weighted RK4 of the tracers): provisional tracers
     (h(1) tr(1) + substep * tend) / hProvis, accumulation of h(1) tr(1) + sum of weight * tend,
     divided by h(2) at the end */
  const int adv = IS(config_advect_tracers) != 0 && nT > 0;
  double *t1 = NULL, *tP = NULL, *t2 = NULL, *tt = R(tend_tracer);
  if (adv) {
    t1 = dalloc((size_t)nT * nC); tP = dalloc((size_t)nT * nC); t2 = dalloc((size_t)nT * nC);
    for (int i = 0; i < nT * nC; i++) t1[i] = tP[i] = A2(R(tracers), 2, 1, i + 1);
    for (int c = 0; c < nC; c++)
      for (int t = 0; t < nT; t++) t2[t + nT * c] = t1[t + nT * c] * h1[c];
  }
  rk_weights[0] = dt / 6.; rk_weights[1] = dt / 3.; rk_weights[2] = dt / 3.; rk_weights[3] = dt / 6.;
  rk_substep_weights[0] = dt / 2.; rk_substep_weights[1] = dt / 2.; rk_substep_weights[2] = dt;
  rk_substep_weights[3] = 0.;
  for (int rk = 1; rk <= 4; rk++) {
    IS(rk_step) = rk;
    TEND_FWD(hP, uP);
    if (adv) scalar_tend_fwd(m, uP, R(h_edge), tP, tt);
    if (rk < 4) {
      for (int e = 0; e < nE; e++) uP[e] = u1[e] + rk_substep_weights[rk - 1] * tu[e];
      for (int c = 0; c < nC; c++) hP[c] = h1[c] + rk_substep_weights[rk - 1] * th[c];
      if (adv)
        for (int c = 0; c < nC; c++)
          for (int t = 0; t < nT; t++)
            tP[t + nT * c] = (h1[c] * t1[t + nT * c] + rk_substep_weights[rk - 1] * tt[t + nT * c]) / hP[c];
    }
    if (IS(config_test_case) == 1) memcpy(uP, u1, sizeof(double) * nE);
    DIAG_FWD(hP, uP);
    for (int e = 0; e < nE; e++) u2[e] = u2[e] + rk_weights[rk - 1] * tu[e];
    for (int c = 0; c < nC; c++) h2[c] = h2[c] + rk_weights[rk - 1] * th[c];
    if (adv)
      for (int i = 0; i < nT * nC; i++) t2[i] = t2[i] + rk_weights[rk - 1] * tt[i];
  }
  if (adv) {
    for (int c = 0; c < nC; c++)
      for (int t = 0; t < nT; t++) A2(R(tracers), 2, 2, t + nT * c + 1) = t2[t + nT * c] / h2[c];
    free(t1); free(tP); free(t2);
  }
  if (IS(config_test_case) == 1) memcpy(u2, u1, sizeof(double) * nE);
  DIAG_FWD(h2, u2);
  RECON(u2);
  put_level(R(u), nE, 2, u2);
  put_level(R(h), nC, 2, h2);
  put_level(R(u), nE, 1, u2);
  put_level(R(h), nC, 1, h2);
  for (int i = 0; i < nT * nC; i++) A2(R(tracers), 2, 1, i + 1) = A2(R(tracers), 2, 2, i + 1);
  free(uP); free(hP); free(u1); free(h1); free(u2); free(h2);
  return 0;
}

int orc_sw_rk4_tlm(orc_mod *m) { /* :637-781 */
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  const double dt = RS(config_dt);
  double rkw[4], rks[4];
  double *uP = dalloc(nE), *hP = dalloc(nC), *uPt = dalloc(nE), *hPt = dalloc(nC);
  double *u1 = dalloc(nE), *h1 = dalloc(nC), *u1t = dalloc(nE), *h1t = dalloc(nC);
  double *u2 = dalloc(nE), *h2 = dalloc(nC), *u2t = dalloc(nE), *h2t = dalloc(nC);
  double *tu = R(tend_u), *th = R(tend_h), *tut = R(tend_u_tl), *tht = R(tend_h_tl);
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  get_level(R(h_tl), nC, 1, h1t); get_level(R(u_tl), nE, 1, u1t);
  diag_tlm(m, dt, h1, h1t, u1, u1t);
  reconstruct_tlm(m, u1, u1t);
  memcpy(uPt, u1t, sizeof(double) * nE); memcpy(uP, u1, sizeof(double) * nE);
  memcpy(hPt, h1t, sizeof(double) * nC); memcpy(hP, h1, sizeof(double) * nC);
  memcpy(u2t, u1t, sizeof(double) * nE); memcpy(u2, u1, sizeof(double) * nE);
  memcpy(h2t, h1t, sizeof(double) * nC); memcpy(h2, h1, sizeof(double) * nC);
  rkw[0] = dt / 6.; rkw[1] = dt / 3.; rkw[2] = dt / 3.; rkw[3] = dt / 6.;
  rks[0] = dt / 2.; rks[1] = dt / 2.; rks[2] = dt; rks[3] = 0.;
  for (int rk = 1; rk <= 4; rk++) {
    IS(rk_step) = rk;
    tend_tlm(m, hP, hPt, uP, uPt);
    if (rk < 4) {
      for (int e = 0; e < nE; e++) uPt[e] = u1t[e] + rks[rk - 1] * tut[e];
      for (int e = 0; e < nE; e++) uP[e] = u1[e] + rks[rk - 1] * tu[e];
      for (int c = 0; c < nC; c++) hPt[c] = h1t[c] + rks[rk - 1] * tht[c];
      for (int c = 0; c < nC; c++) hP[c] = h1[c] + rks[rk - 1] * th[c];
    }
    if (IS(config_test_case) == 1) {
      memcpy(uPt, u1t, sizeof(double) * nE);
      memcpy(uP, u1, sizeof(double) * nE);
    }
    diag_tlm(m, dt, hP, hPt, uP, uPt);
    for (int e = 0; e < nE; e++) u2t[e] = u2t[e] + rkw[rk - 1] * tut[e];
    for (int e = 0; e < nE; e++) u2[e] = u2[e] + rkw[rk - 1] * tu[e];
    for (int c = 0; c < nC; c++) h2t[c] = h2t[c] + rkw[rk - 1] * tht[c];
    for (int c = 0; c < nC; c++) h2[c] = h2[c] + rkw[rk - 1] * th[c];
  }
  if (IS(config_test_case) == 1) {
    memcpy(u2t, u1t, sizeof(double) * nE);
    memcpy(u2, u1, sizeof(double) * nE);
  }
  diag_tlm(m, dt, h2, h2t, u2, u2t);
  reconstruct_tlm(m, u2, u2t);
  put_level(R(u_tl), nE, 2, u2t); put_level(R(u), nE, 2, u2);
  put_level(R(h_tl), nC, 2, h2t); put_level(R(h), nC, 2, h2);
  put_level(R(u_tl), nE, 1, u2t); put_level(R(u), nE, 1, u2);
  put_level(R(h_tl), nC, 1, h2t); put_level(R(h), nC, 1, h2);
  free(uP); free(hP); free(uPt); free(hPt); free(u1); free(h1); free(u1t); free(h1t);
  free(u2); free(h2); free(u2t); free(h2t);
  return 0;
}

int orc_sw_rk4_adj(orc_mod *m) { /* :783-1002 */
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  const double dt = RS(config_dt);
  double rkw[4], rks[4];
  double *uP = dalloc((size_t)5 * nE), *hP = dalloc((size_t)5 * nC);   /* uProvis(5,1,nEdges) */
  double *uPa = dalloc(nE), *hPa = dalloc(nC);
  double *u1 = dalloc(nE), *h1 = dalloc(nC), *u2 = dalloc(nE), *h2 = dalloc(nC);
  double *u1a = dalloc(nE), *h1a = dalloc(nC), *u2a = dalloc(nE), *h2a = dalloc(nC);
  double *tu = R(tend_u), *th = R(tend_h), *tua = R(tend_u_ad), *tha = R(tend_h_ad);
#define UP(k) (uP + (size_t)((k) - 1) * nE)
#define HP(k) (hP + (size_t)((k) - 1) * nC)
  for (int e = 0; e < nE; e++) uPa[e] = 0.;
  for (int c = 0; c < nC; c++) hPa[c] = 0.;
  rkw[0] = dt / 6.; rkw[1] = dt / 3.; rkw[2] = dt / 3.; rkw[3] = dt / 6.;
  rks[0] = dt / 2.; rks[1] = dt / 2.; rks[2] = dt; rks[3] = 0.;

  /* forward sweep :815-878 */
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  DIAG_FWD(h1, u1);
  RECON(u1);
  memcpy(UP(1), u1, sizeof(double) * nE);
  memcpy(HP(1), h1, sizeof(double) * nC);
  memcpy(u2, u1, sizeof(double) * nE);
  memcpy(h2, h1, sizeof(double) * nC);
  for (int rk = 1; rk <= 4; rk++) {
    IS(rk_step) = rk;
    TEND_FWD(HP(rk), UP(rk));
    if (rk < 4) {
      for (int e = 0; e < nE; e++) UP(rk + 1)[e] = u1[e] + rks[rk - 1] * tu[e];
      for (int c = 0; c < nC; c++) HP(rk + 1)[c] = h1[c] + rks[rk - 1] * th[c];
    } else {
      memcpy(UP(rk + 1), UP(rk), sizeof(double) * nE);
      memcpy(HP(rk + 1), HP(rk), sizeof(double) * nC);
    }
    if (IS(config_test_case) == 1) memcpy(UP(rk + 1), u1, sizeof(double) * nE);
    DIAG_FWD(HP(rk + 1), UP(rk + 1));
    for (int e = 0; e < nE; e++) u2[e] = u2[e] + rkw[rk - 1] * tu[e];
    for (int c = 0; c < nC; c++) h2[c] = h2[c] + rkw[rk - 1] * th[c];
  }
  put_level(R(u), nE, 2, u2);
  put_level(R(h), nC, 2, h2);

  /* :882-885 */
  get_level(R(h_ad), nC, 1, h2a);
  for (int c = 0; c < nC; c++) h1a[c] = 0;
  get_level(R(u_ad), nE, 1, u2a);
  for (int e = 0; e < nE; e++) u1a[e] = 0;

  reconstruct_adj(m, u2a);                                  /* :887-892 */
  diag_adj(m, dt, h2, h2a, u2, u2a);                         /* :894-905 */
  if (IS(config_test_case) == 1) {                          /* :907-910 */
    for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + u2a[e];
    for (int e = 0; e < nE; e++) u2a[e] = 0.;
  }
  for (int rk = 4; rk >= 1; rk--) {                         /* :912-970 */
    IS(rk_step) = rk;
    for (int c = 0; c < nC; c++) tha[c] = tha[c] + rkw[rk - 1] * h2a[c];
    for (int e = 0; e < nE; e++) tua[e] = tua[e] + rkw[rk - 1] * u2a[e];
    diag_adj(m, dt, HP(rk + 1), hPa, UP(rk + 1), uPa);
    if (IS(config_test_case) == 1) {
      for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + uPa[e];
      for (int e = 0; e < nE; e++) uPa[e] = 0.;
    }
    if (rk < 4) {
      for (int c = 0; c < nC; c++) tha[c] = tha[c] + rks[rk - 1] * hPa[c];
      for (int c = 0; c < nC; c++) h1a[c] = h1a[c] + hPa[c];
      for (int c = 0; c < nC; c++) hPa[c] = 0.;
      for (int e = 0; e < nE; e++) tua[e] = tua[e] + rks[rk - 1] * uPa[e];
      for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + uPa[e];
      for (int e = 0; e < nE; e++) uPa[e] = 0.;
    }
    DIAG_FWD(HP(rk), UP(rk));
    tend_adj(m, HP(rk), hPa, UP(rk), uPa);
  }
  for (int c = 0; c < nC; c++) h1a[c] = h1a[c] + h2a[c];    /* :972-980 */
  for (int c = 0; c < nC; c++) h2a[c] = 0.;
  for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + u2a[e];
  for (int e = 0; e < nE; e++) u2a[e] = 0.;
  for (int c = 0; c < nC; c++) h1a[c] = h1a[c] + hPa[c];
  for (int c = 0; c < nC; c++) hPa[c] = 0.;
  for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + uPa[e];
  for (int e = 0; e < nE; e++) uPa[e] = 0.;
  reconstruct_adj(m, u1a);                                  /* :982-987 */
  diag_adj(m, dt, h1, h1a, u1, u1a);                        /* :989-1000 */
  put_level(R(h_ad), nC, 1, h1a); put_level(R(h_ad), nC, 2, h2a);
  put_level(R(u_ad), nE, 1, u1a); put_level(R(u_ad), nE, 2, u2a);
#undef UP
#undef HP
  free(uP); free(hP); free(uPa); free(hPa); free(u1); free(h1); free(u2); free(h2);
  free(u1a); free(h1a); free(u2a); free(h2a);
  return 0;
}

static double sumsq(const double *x, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; i++) s = s + x[i] * x[i];
  return s;
}

int orc_link_tlm_adj(orc_mod *m, int print) { /* :1006-1218 (returns instead of STOP) */
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges), nV = IS(nVertices);
  const double dt = RS(config_dt);
  double rks[4];
  double *uPf = dalloc(nE), *hPf = dalloc(nC);   /* uProvis_fw(1,:,:) (only stage 1 used) */
  double *uP = dalloc(nE), *hP = dalloc(nC), *uPt = dalloc(nE), *hPt = dalloc(nC);
  double *uPa = dalloc(nE), *hPa = dalloc(nC);
  double *u1 = dalloc(nE), *h1 = dalloc(nC), *u1t = dalloc(nE), *h1t = dalloc(nC);
  double *u2t = dalloc(nE), *h2t = dalloc(nC), *u1a = dalloc(nE), *h1a = dalloc(nC),
         *u2a = dalloc(nE), *h2a = dalloc(nC);
  RS(pt) = 1.E-3;
  rks[0] = dt / 2.; rks[1] = dt / 2.; rks[2] = dt; rks[3] = 0.;
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  get_level(R(h_tl), nC, 1, h1t); get_level(R(u_tl), nE, 1, u1t);
  diag_tlm(m, dt, h1, h1t, u1, u1t);
  reconstruct_tlm(m, u1, u1t);
  memcpy(uPt, u1t, sizeof(double) * nE); memcpy(uP, u1, sizeof(double) * nE);
  memcpy(uPf, u1, sizeof(double) * nE);
  memcpy(hPt, h1t, sizeof(double) * nC); memcpy(hP, h1, sizeof(double) * nC);
  memcpy(hPf, h1, sizeof(double) * nC);
  memcpy(u2t, u1t, sizeof(double) * nE); memcpy(h2t, h1t, sizeof(double) * nC);
  put_level(R(u), nE, 2, u1); put_level(R(h), nC, 2, h1);
  {
    const int rk = 1;
    IS(rk_step) = rk;
    tend_tlm(m, hP, hPt, uP, uPt);
    for (int e = 0; e < nE; e++) uPt[e] = u1t[e] + rks[rk - 1] * R(tend_u_tl)[e];
    for (int e = 0; e < nE; e++) uP[e] = u1[e] + rks[rk - 1] * R(tend_u)[e];
    for (int c = 0; c < nC; c++) hPt[c] = h1t[c] + rks[rk - 1] * R(tend_h_tl)[c];
    for (int c = 0; c < nC; c++) hP[c] = h1[c] + rks[rk - 1] * R(tend_h)[c];
  }
  /* :1090-1110 */
  double LHS = sumsq(uPt, nE) + sumsq(hPt, nC) + sumsq(R(tend_h_tl), nC) + sumsq(R(tend_u_tl), nE) +
               sumsq(u2t, nE) + sumsq(h2t, nC) + sumsq(R(v_tl), nE) + sumsq(R(h_edge_tl), nE) +
               sumsq(R(h_vertex_tl), nV) + sumsq(R(circulation_tl), nV) + sumsq(R(vorticity_tl), nV) +
               sumsq(R(divergence_tl), nC) + sumsq(R(ke_tl), nC) + sumsq(R(pv_edge_tl), nE) +
               sumsq(R(pv_vertex_tl), nV) + sumsq(R(pv_cell_tl), nC) + sumsq(R(vorticity_cell_tl), nC) +
               sumsq(R(gradPVn_tl), nE) + sumsq(R(gradPVt_tl), nE) + sumsq(R(uReconstructX_tl), nC) +
               sumsq(R(uReconstructY_tl), nC) + sumsq(R(uReconstructZ_tl), nC) +
               sumsq(R(uReconstructZonal_tl), nC) + sumsq(R(uReconstructMeridional_tl), nC);
  /* :1112-1135 */
  memcpy(uPa, uPt, sizeof(double) * nE); memcpy(hPa, hPt, sizeof(double) * nC);
  memcpy(R(tend_h_ad), R(tend_h_tl), sizeof(double) * nC);
  memcpy(R(tend_u_ad), R(tend_u_tl), sizeof(double) * nE);
  memcpy(u2a, u2t, sizeof(double) * nE); memcpy(h2a, h2t, sizeof(double) * nC);
  get_level(R(h_ad), nC, 1, h1a); get_level(R(u_ad), nE, 1, u1a);
#define CP(dst, src, n) memcpy(R(dst), R(src), sizeof(double) * (n))
  CP(v_ad, v_tl, nE); CP(h_edge_ad, h_edge_tl, nE); CP(h_vertex_ad, h_vertex_tl, nV);
  CP(circulation_ad, circulation_tl, nV); CP(vorticity_ad, vorticity_tl, nV);
  CP(divergence_ad, divergence_tl, nC); CP(ke_ad, ke_tl, nC); CP(pv_edge_ad, pv_edge_tl, nE);
  CP(pv_vertex_ad, pv_vertex_tl, nV); CP(pv_cell_ad, pv_cell_tl, nC);
  CP(vorticity_cell_ad, vorticity_cell_tl, nC); CP(gradPVn_ad, gradPVn_tl, nE);
  CP(gradPVt_ad, gradPVt_tl, nE); CP(uReconstructX_ad, uReconstructX_tl, nC);
  CP(uReconstructY_ad, uReconstructY_tl, nC); CP(uReconstructZ_ad, uReconstructZ_tl, nC);
  CP(uReconstructZonal_ad, uReconstructZonal_tl, nC);
  CP(uReconstructMeridional_ad, uReconstructMeridional_tl, nC);
#undef CP
  {
    const int rk = 1; /* :1139-1176 */
    for (int c = 0; c < nC; c++) R(tend_h_ad)[c] = R(tend_h_ad)[c] + rks[rk - 1] * hPa[c];
    for (int c = 0; c < nC; c++) h1a[c] = h1a[c] + hPa[c];
    for (int c = 0; c < nC; c++) hPa[c] = 0.;
    for (int e = 0; e < nE; e++) R(tend_u_ad)[e] = R(tend_u_ad)[e] + rks[rk - 1] * uPa[e];
    for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + uPa[e];
    for (int e = 0; e < nE; e++) uPa[e] = 0.;
    DIAG_FWD(hPf, uPf);
    tend_adj(m, hPf, hPa, uPf, uPa);
  }
  for (int c = 0; c < nC; c++) h1a[c] = h1a[c] + h2a[c];
  for (int c = 0; c < nC; c++) h2a[c] = 0.;
  for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + u2a[e];
  for (int e = 0; e < nE; e++) u2a[e] = 0.;
  for (int c = 0; c < nC; c++) h1a[c] = h1a[c] + hPa[c];
  for (int e = 0; e < nE; e++) u1a[e] = u1a[e] + uPa[e];
  reconstruct_adj(m, u1a);
  diag_adj(m, dt, h1, h1a, u1, u1a);
  put_level(R(h_ad), nC, 1, h1a); put_level(R(h_ad), nC, 2, h2a);
  put_level(R(u_ad), nE, 1, u1a); put_level(R(u_ad), nE, 2, u2a);
  double RHS = 0.0, s2 = 0.0;
  for (int e = 0; e < nE; e++) RHS = RHS + u1a[e] * u1[e] * RS(pt);
  for (int c = 0; c < nC; c++) s2 = s2 + h1a[c] * h1[c] * RS(pt);
  RHS = RHS + s2;
  RS(LHS) = LHS;
  RS(RHS) = RHS;
  if (print) {
    printf("%25.16E\n%25.16E\n%25.16E\n%25.16E\n", LHS, RHS, (LHS - RHS) / LHS, (LHS - RHS) / RHS);
    fflush(stdout);
  }
  free(uPf); free(hPf); free(uP); free(hP); free(uPt); free(hPt); free(uPa); free(hPa);
  free(u1); free(h1); free(u1t); free(h1t); free(u2t); free(h2t); free(u1a); free(h1a);
  free(u2a); free(h2a);
  return 0;
}

/* single-call entry points for per-routine parity */
int orc_solve_diagnostics(orc_mod *m) {
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  const double dt = RS(config_dt);
  double *h1 = dalloc(nC), *u1 = dalloc(nE);
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  DIAG_FWD(h1, u1);
  free(h1); free(u1);
  return 0;
}
int orc_compute_tend(orc_mod *m) {
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  double *h1 = dalloc(nC), *u1 = dalloc(nE);
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  TEND_FWD(h1, u1);
  free(h1); free(u1);
  return 0;
}
int orc_solve_diagnostics_tlm(orc_mod *m) {
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  double *h1 = dalloc(nC), *u1 = dalloc(nE), *h1t = dalloc(nC), *u1t = dalloc(nE);
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  get_level(R(h_tl), nC, 1, h1t); get_level(R(u_tl), nE, 1, u1t);
  diag_tlm(m, RS(config_dt), h1, h1t, u1, u1t);
  free(h1); free(u1); free(h1t); free(u1t);
  return 0;
}
int orc_compute_tend_tlm(orc_mod *m) {
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  double *h1 = dalloc(nC), *u1 = dalloc(nE), *h1t = dalloc(nC), *u1t = dalloc(nE);
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  get_level(R(h_tl), nC, 1, h1t); get_level(R(u_tl), nE, 1, u1t);
  tend_tlm(m, h1, h1t, u1, u1t);
  free(h1); free(u1); free(h1t); free(u1t);
  return 0;
}
int orc_solve_diagnostics_adj(orc_mod *m) {
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  double *h1 = dalloc(nC), *u1 = dalloc(nE), *h1a = dalloc(nC), *u1a = dalloc(nE);
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  get_level(R(h_ad), nC, 1, h1a); get_level(R(u_ad), nE, 1, u1a);
  diag_adj(m, RS(config_dt), h1, h1a, u1, u1a);
  put_level(R(h_ad), nC, 1, h1a); put_level(R(u_ad), nE, 1, u1a);
  free(h1); free(u1); free(h1a); free(u1a);
  return 0;
}
int orc_compute_tend_adj(orc_mod *m) {
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges);
  double *h1 = dalloc(nC), *u1 = dalloc(nE), *h1a = dalloc(nC), *u1a = dalloc(nE);
  get_level(R(h), nC, 1, h1); get_level(R(u), nE, 1, u1);
  get_level(R(h_ad), nC, 1, h1a); get_level(R(u_ad), nE, 1, u1a);
  tend_adj(m, h1, h1a, u1, u1a);
  put_level(R(h_ad), nC, 1, h1a); put_level(R(u_ad), nE, 1, u1a);
  free(h1); free(u1); free(h1a); free(u1a);
  return 0;
}
int orc_compute_scalar_tend(orc_mod *m) {
  if (check(m)) return 1;
  const int nC = IS(nCells), nE = IS(nEdges), nT = IS(nTracers);
  double *u1 = dalloc(nE), *t1 = dalloc((size_t)nT * nC + 1);
  get_level(R(u), nE, 1, u1);
  for (int i = 0; i < nT * nC; i++) t1[i] = A2(R(tracers), 2, 1, i + 1);
  scalar_tend_fwd(m, u1, R(h_edge), t1, R(tend_tracer));
  free(u1); free(t1);
  return 0;
}

int orc_reconstruct_2d(orc_mod *m) {
  if (check(m)) return 1;
  const int nE = IS(nEdges);
  double *u1 = dalloc(nE);
  get_level(R(u), nE, 1, u1);
  RECON(u1);
  free(u1);
  return 0;
}

/* ---------------------------------------------------------------------------------------- */
/* Williamson test cases: src/mpas_sw_testcases.f90                                           */
/* ---------------------------------------------------------------------------------------- */
static double sphere_distance(double lat1, double lon1, double lat2, double lon2, double radius) {
  const double s1 = sin(0.5 * (lat2 - lat1)), s2 = sin(0.5 * (lon2 - lon1));
  const double arg1 = sqrt(s1 * s1 + cos(lat1) * cos(lat2) * (s2 * s2));
  return 2. * radius * asin(arg1);
}

static void scale_to_earth(orc_mod *m) { /* e.g. :173-186 */
  const int nC = IS(nCells), nE = IS(nEdges), nV = IS(nVertices), vd = IS(vertexDegree);
  for (int i = 0; i < nC; i++) { R(xCell)[i] *= A_EARTH; R(yCell)[i] *= A_EARTH; R(zCell)[i] *= A_EARTH; }
  for (int i = 0; i < nV; i++) { R(xVertex)[i] *= A_EARTH; R(yVertex)[i] *= A_EARTH; R(zVertex)[i] *= A_EARTH; }
  for (int i = 0; i < nE; i++) { R(xEdge)[i] *= A_EARTH; R(yEdge)[i] *= A_EARTH; R(zEdge)[i] *= A_EARTH; }
  for (int i = 0; i < nE; i++) { R(dvEdge)[i] = R(dvEdge)[i] * A_EARTH; R(dcEdge)[i] = R(dcEdge)[i] * A_EARTH; }
  const double a2 = A_EARTH * A_EARTH;
  for (int i = 0; i < nC; i++) R(areaCell)[i] = R(areaCell)[i] * a2;
  for (int i = 0; i < nV; i++) R(areaTriangle)[i] = R(areaTriangle)[i] * a2;
  for (int i = 0; i < nV * vd; i++) R(kiteAreasOnVertex)[i] = R(kiteAreasOnVertex)[i] * a2;
}

static void wind_from_psi(orc_mod *m, const double *psiVertex) {
  for (int e = 1; e <= IS(nEdges); e++)
    A2(R(u), 2, 1, e) = -1.0 * (A1(psiVertex, A2(I(verticesOnEdge), 2, 2, e)) -
                                A1(psiVertex, A2(I(verticesOnEdge), 2, 1, e))) / A1(R(dvEdge), e);
}

static void coriolis(orc_mod *m, double alpha) {
  for (int e = 1; e <= IS(nEdges); e++)
    A1(R(fEdge), e) = 2.0 * OMEGA * (-cos(A1(R(lonEdge), e)) * cos(A1(R(latEdge), e)) * sin(alpha) +
                                     sin(A1(R(latEdge), e)) * cos(alpha));
  for (int v = 1; v <= IS(nVertices); v++)
    A1(R(fVertex), v) = 2.0 * OMEGA * (-cos(A1(R(lonVertex), v)) * cos(A1(R(latVertex), v)) * sin(alpha) +
                                       sin(A1(R(latVertex), v)) * cos(alpha));
}

int orc_sw_test_case_1(orc_mod *m) { /* :1-66 */
  const double u0 = 2.0 * PII * A_EARTH / (12.0 * 86400.0), h0 = 1000.0, theta_c = 0.0;
  const double lambda_c = 3.0 * PII / 2.0, alpha = PII / 4.0;
  scale_to_earth(m);
  double *psi = dalloc(IS(nVertices));
  for (int v = 1; v <= IS(nVertices); v++)
    A1(psi, v) = -A_EARTH * u0 * (sin(A1(R(latVertex), v)) * cos(alpha) -
                                  cos(A1(R(lonVertex), v)) * cos(A1(R(latVertex), v)) * sin(alpha));
  wind_from_psi(m, psi);
  free(psi);
  for (int c = 1; c <= IS(nCells); c++) {
    const double r = sphere_distance(theta_c, lambda_c, A1(R(latCell), c), A1(R(lonCell), c), A_EARTH);
    if (r < A_EARTH / 3.0) A2(R(h), 2, 1, c) = (h0 / 2.0) * (1.0 + cos(PII * r * 3.0 / A_EARTH));
    else A2(R(h), 2, 1, c) = h0 / 2.0;
  }
  return 0;
}

int orc_sw_test_case_2(orc_mod *m) { /* :68-145 */
  const double u0 = 2.0 * PII * A_EARTH / (12.0 * 86400.0), gh0 = 29400.0, alpha = 0.0;
  scale_to_earth(m);
  double *psi = dalloc(IS(nVertices));
  for (int v = 1; v <= IS(nVertices); v++)
    A1(psi, v) = -A_EARTH * u0 * (sin(A1(R(latVertex), v)) * cos(alpha) -
                                  cos(A1(R(lonVertex), v)) * cos(A1(R(latVertex), v)) * sin(alpha));
  wind_from_psi(m, psi);
  free(psi);
  coriolis(m, alpha);
  for (int c = 1; c <= IS(nCells); c++) {
    const double x = -cos(A1(R(lonCell), c)) * cos(A1(R(latCell), c)) * sin(alpha) +
                     sin(A1(R(latCell), c)) * cos(alpha);
    A2(R(h), 2, 1, c) = (gh0 - (A_EARTH * OMEGA * u0 + 0.5 * (u0 * u0)) * (x * x)) / GRAVITY;
  }
  return 0;
}

int orc_sw_test_case_5(orc_mod *m) { /* :147-254 */
  const double u0 = 20., gh0 = 5960.0 * GRAVITY, hs0 = 2000., theta_c = PII / 6.0;
  const double lambda_c = 3.0 * PII / 2.0, rr = PII / 9.0, alpha = 0.0;
  scale_to_earth(m);
  double *psi = dalloc(IS(nVertices));
  for (int v = 1; v <= IS(nVertices); v++)
    A1(psi, v) = -A_EARTH * u0 * (sin(A1(R(latVertex), v)) * cos(alpha) -
                                  cos(A1(R(lonVertex), v)) * cos(A1(R(latVertex), v)) * sin(alpha));
  wind_from_psi(m, psi);
  free(psi);
  coriolis(m, alpha);
  for (int c = 1; c <= IS(nCells); c++) {
    if (A1(R(lonCell), c) < 0.0) A1(R(lonCell), c) = A1(R(lonCell), c) + 2.0 * PII;
    const double dl = A1(R(lonCell), c) - lambda_c, dp = A1(R(latCell), c) - theta_c;
    const double r = sqrt(fmin(rr * rr, dl * dl + dp * dp));
    A1(R(h_s), c) = hs0 * (1.0 - r / rr);
  }
  for (int c = 1; c <= IS(nCells); c++) {
    const double dl = A1(R(lonCell), c) - lambda_c, dp = A1(R(latCell), c) - theta_c;
    const double r = sqrt(fmin(rr * rr, dl * dl + dp * dp));
    if (IS(nTracers) >= 1) R(tracers)[2 * (c - 1) * IS(nTracers)] = 1.0 - r / rr;
  }
  for (int c = 1; c <= IS(nCells); c++) {
    const double x = -cos(A1(R(lonCell), c)) * cos(A1(R(latCell), c)) * sin(alpha) +
                     sin(A1(R(latCell), c)) * cos(alpha);
    A2(R(h), 2, 1, c) = (gh0 - (A_EARTH * OMEGA * u0 + 0.5 * (u0 * u0)) * (x * x)) / GRAVITY;
    A2(R(h), 2, 1, c) = A2(R(h), 2, 1, c) - A1(R(h_s), c);
  }
  return 0;
}

static const double RH_W = 7.848e-6, RH_K = 7.848e-6, RH_R = 4.0;
static double rh_aa(double theta) { /* :341-360 */
  const double c = cos(theta);
  return 0.5 * RH_W * (2.0 * OMEGA + RH_W) * (c * c) +
         0.25 * (RH_K * RH_K) * pow(c, 2.0 * RH_R) *
             ((RH_R + 1.0) * (c * c) + 2.0 * (RH_R * RH_R) - RH_R - 2.0 - 2.0 * (RH_R * RH_R) * pow(c, -2.0));
}
static double rh_bb(double theta) { /* :362-379 */
  const double c = cos(theta);
  return (2.0 * (OMEGA + RH_W) * RH_K / ((RH_R + 1.0) * (RH_R + 2.0))) * pow(c, RH_R) *
         (((RH_R * RH_R) + 2.0 * RH_R + 2.0) - ((RH_R + 1.0) * c) * ((RH_R + 1.0) * c));
}
static double rh_cc(double theta) { /* :381-398 */
  const double c = cos(theta);
  return 0.25 * (RH_K * RH_K) * pow(c, 2.0 * RH_R) * ((RH_R + 1.0) * (c * c) - RH_R - 2.0);
}

int orc_sw_test_case_6(orc_mod *m) { /* :256-319 (leaves fEdge/fVertex untouched, as the reference) */
  const double h0 = 8000.0;
  scale_to_earth(m);
  double *psi = dalloc(IS(nVertices));
  for (int v = 1; v <= IS(nVertices); v++) {
    const double lat = A1(R(latVertex), v), lon = A1(R(lonVertex), v);
    A1(psi, v) = -A_EARTH * A_EARTH * RH_W * sin(lat) +
                 A_EARTH * A_EARTH * RH_K * pow(cos(lat), RH_R) * sin(lat) * cos(RH_R * lon);
  }
  wind_from_psi(m, psi);
  free(psi);
  for (int c = 1; c <= IS(nCells); c++) {
    const double lat = A1(R(latCell), c), lon = A1(R(lonCell), c);
    A2(R(h), 2, 1, c) = (GRAVITY * h0 + A_EARTH * A_EARTH * rh_aa(lat) +
                         A_EARTH * A_EARTH * rh_bb(lat) * cos(RH_R * lon) +
                         A_EARTH * A_EARTH * rh_cc(lat) * cos(2.0 * RH_R * lon)) / GRAVITY;
  }
  return 0;
}
