// Host set-up of the engine: mesh validation, space-filling-curve renumbering, transposed
// gather lists, and the once-per-run geometry of sw_mpas_init_block
// (src/mpas_sw_module.f90:495-526): mesh scaling, unit vectors and RBF reconstruction
// coefficients.
#pragma once

#include <string>
#include <vector>

namespace mpsw {

// Mesh arrays exactly as the reference module holds them: Fortran column-major, 1-based.
struct RefMesh {
  int nC = 0, nE = 0, nV = 0, maxEdges = 0, maxEdges2 = 0, vd = 0;
  const int *cellsOnEdge = nullptr, *verticesOnEdge = nullptr, *edgesOnEdge = nullptr,
            *nEdgesOnEdge = nullptr, *edgesOnCell = nullptr, *nEdgesOnCell = nullptr,
            *cellsOnVertex = nullptr, *edgesOnVertex = nullptr;
  const double *weightsOnEdge = nullptr, *kiteAreasOnVertex = nullptr, *dcEdge = nullptr,
               *dvEdge = nullptr, *areaCell = nullptr, *areaTriangle = nullptr,
               *fVertex = nullptr, *h_s = nullptr, *u_src = nullptr, *meshDensity = nullptr;
  const double *xCell = nullptr, *yCell = nullptr, *zCell = nullptr, *xEdge = nullptr,
               *yEdge = nullptr, *zEdge = nullptr, *xVertex = nullptr, *yVertex = nullptr,
               *zVertex = nullptr, *latCell = nullptr, *lonCell = nullptr;
  int on_a_sphere = 1, h_ScaleWithMesh = 0;
};

// Derived geometry, reference layout (module variables written by sw_mpas_init_block).
struct RefGeometry {
  std::vector<double> meshScalingDel2, meshScalingDel4;     // (nEdges)
  std::vector<double> localVerticalUnitVectors;             // (3, nCells)
  std::vector<double> edgeNormalVectors;                    // (3, nEdges)
  std::vector<double> cellTangentPlane;                     // (3, 2, nCells)
  std::vector<double> coeffs_reconstruct;                   // (3, maxEdges, nCells)
};

// Internal-order mesh, slot-major, 0-based (see mpsw_internal.h for the meaning of fields).
struct BuiltMesh {
  int nC = 0, nE = 0, nV = 0;
  std::vector<int> perm_c, perm_e, perm_v;  // reference index -> internal index
  std::vector<int> c_n, c_eoc, c_es, c_vs;
  std::vector<signed char> c_esg, v_esg;
  std::vector<double> c_vk, c_area, c_hs, c_coef, c_trig;
  std::vector<int> e_c1, e_c2, e_v1, e_v2, e_va, e_vb, e_slot1, e_slot2, e_n, e_eoe, e_rev;
  std::vector<double> e_w, e_wrev, e_dc, e_dv, e_sc2, e_sc4, e_usrc;
  std::vector<int> v_es, v_c, v_e;
  std::vector<double> v_k, v_area, v_f;
};

// Check every index and count; empty string on success, else the first problem found.
std::string validate_mesh(const RefMesh &m);

// Geometry of sw_mpas_init_block: compute_mesh_scaling (src/mpas_sw_dyncore.f90:363-393),
// mpas_initialize_vectors and mpas_init_reconstruct (src/mpas_sw_operators.f90:2-279).
void compute_geometry(const RefMesh &m, RefGeometry *g);

// Renumber (Hilbert order when sfc != 0, identity otherwise) and build the gather lists.
std::string build_mesh(const RefMesh &m, const RefGeometry &g, int sfc, BuiltMesh *out);

}  // namespace mpsw
