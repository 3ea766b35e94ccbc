// extern "C" wrappers around the reference's own generated kernels and FEniCS form, compiled
// from the reference sources into oracle/_ref/libhyteg_ref.so by oracle/Makefile.
// TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle and the product against the
// reference implementation; never linked into the product.
#include <cstdint>
#include <map>

#include "hyteg/fenics/ufc.h"
#include "hyteg/forms/form_fenics_generated/p1_tet_diffusion.h"
#include "hyteg/forms/form_fenics_generated/p1_tet_mass.h"
#include "hyteg/forms/form_fenics_generated/p1_tet_pspg_tet.h"
#include "hyteg/forms/form_fenics_generated/p2_tet_diffusion.h"
#include "hyteg/forms/form_fenics_generated/p2_to_p1_tet_div_tet.h"
#include "hyteg/forms/form_fenics_generated/p1_to_p2_tet_divt_tet.h"
#include "hyteg/gridtransferoperators/generatedKernels/prolongate_3D_macrocell_P1_push_additive.hpp"
#include "hyteg/gridtransferoperators/generatedKernels/restrict_3D_macrocell_P1_pull_additive.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macrocell_vertexdof_to_vertexdof_add.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macrocell_vertexdof_to_vertexdof_replace.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macroface_one_sided_vertexdof_to_vertexdof_add.hpp"
#include "hyteg/p1functionspace/generatedKernels/apply_3D_macroface_one_sided_vertexdof_to_vertexdof_replace.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macrocell_P1.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1.hpp"
#include "hyteg/p1functionspace/generatedKernels/sor_3D_macroface_P1_one_sided.hpp"

using hyteg::indexing::IndexIncrement;
typedef std::map<IndexIncrement, double> StencilMap;

// The 15 cell-stencil increments in the order C E W N S NW SE TC TW TS TSE BC BE BN BNW.
static const int kOff[15][3] = {{0, 0, 0},  {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
                                {-1, 1, 0}, {1, -1, 0}, {0, 0, 1},  {-1, 0, 1}, {0, -1, 1},
                                {1, -1, 1}, {0, 0, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 1, -1}};

// present == nullptr keeps all 15 increments; otherwise only those with present[k] != 0 (the
// one-sided face stencils contain the increments that stay inside the neighbour cell).
static StencilMap toMap(const double* w, const int* present) {
  StencilMap m;
  for (int k = 0; k < 15; ++k)
    if (!present || present[k]) m[IndexIncrement(kOff[k][0], kOff[k][1], kOff[k][2])] = w[k];
  return m;
}

extern "C" {

void ref_apply_cell(double* dst, const double* src, int level, const double* w15, int add) {
  if (add)
    hyteg::vertexdof::macrocell::generated::apply_3D_macrocell_vertexdof_to_vertexdof_add(dst, src, level, toMap(w15, nullptr));
  else
    hyteg::vertexdof::macrocell::generated::apply_3D_macrocell_vertexdof_to_vertexdof_replace(dst, src, level,
                                                                                               toMap(w15, nullptr));
}

void ref_sor_cell(double* dst, const double* rhs, int level, const double* w15, double relax) {
  hyteg::vertexdof::macrocell::generated::sor_3D_macrocell_P1(dst, rhs, level, toMap(w15, nullptr), relax);
}

// One-sided face apply with the ghost layer `srcGl` of a neighbour cell whose cell-local
// vertex IDs of the face's vertices are (v0, v1, v2); w15 = that cell's contribution to the
// face-point row in cell-local increments.
void ref_apply_face(double* dst, const double* src, const double* srcGl, int level, int64_t v0, int64_t v1, int64_t v2,
                    const double* w15, const int* present15, int add) {
  if (add)
    hyteg::vertexdof::macroface::generated::apply_3D_macroface_one_sided_vertexdof_to_vertexdof_add(
        dst, src, srcGl, level, v0, v1, v2, toMap(w15, present15));
  else
    hyteg::vertexdof::macroface::generated::apply_3D_macroface_one_sided_vertexdof_to_vertexdof_replace(
        dst, src, srcGl, level, v0, v1, v2, toMap(w15, present15));
}

void ref_restrict_cell(double* coarse, const double* fine, int coarseLevel, const double* nEdge6, const double* nFace4,
                       const double* nVert4) {
  hyteg::vertexdof::macrocell::generated::restrict_3D_macrocell_P1_pull_additive(
      coarse, fine, coarseLevel, nEdge6[0], nEdge6[1], nEdge6[2], nEdge6[3], nEdge6[4], nEdge6[5], nFace4[0], nFace4[1],
      nFace4[2], nFace4[3], nVert4[0], nVert4[1], nVert4[2], nVert4[3]);
}

void ref_prolongate_cell(const double* coarse, double* fine, int coarseLevel, const double* nEdge6, const double* nFace4,
                         const double* nVert4) {
  hyteg::vertexdof::macrocell::generated::prolongate_3D_macrocell_P1_push_additive(
      coarse, fine, coarseLevel, nEdge6[0], nEdge6[1], nEdge6[2], nEdge6[3], nEdge6[4], nEdge6[5], nFace4[0], nFace4[1],
      nFace4[2], nFace4[3], nVert4[0], nVert4[1], nVert4[2], nVert4[3]);
}

// FEniCS/UFC P1 element matrices of the reference (forms/form_fenics_generated/*.h).
void ref_p1_tet_diffusion(const double* coords12, double* K16) {
  p1_tet_diffusion_cell_integral_0_otherwise f;
  f.tabulate_tensor(K16, nullptr, coords12, 0);
}

void ref_p1_tet_mass(const double* coords12, double* K16) {
  p1_tet_mass_cell_integral_0_otherwise f;
  f.tabulate_tensor(K16, nullptr, coords12, 0);
}

// PSPG stabilisation form -tau grad p . grad q, tau = |T|^(2/3) / 12 (P1PSPGOperator; its
// inverse diagonal is the pressure scaling of the Uzawa smoother).
void ref_p1_tet_pspg(const double* coords12, double* K16) {
  p1_tet_pspg_tet_cell_integral_0_otherwise f;
  f.tabulate_tensor(K16, nullptr, coords12, 0);
}

// Divergence P2 -> P1 (component k; 4 x 10) and its transpose form P1 -> P2 (10 x 4) of the
// reference's FEniCS forms (P2P1TaylorHoodStokesOperator div / divT), UFC local node order.
void ref_p2_to_p1_div(const double* coords12, int k, double* A40) {
  if (k == 0) {
    p2_to_p1_tet_div_tet_cell_integral_0_otherwise f;
    f.tabulate_tensor(A40, nullptr, coords12, 0);
  } else if (k == 1) {
    p2_to_p1_tet_div_tet_cell_integral_1_otherwise f;
    f.tabulate_tensor(A40, nullptr, coords12, 0);
  } else {
    p2_to_p1_tet_div_tet_cell_integral_2_otherwise f;
    f.tabulate_tensor(A40, nullptr, coords12, 0);
  }
}

void ref_p1_to_p2_divt(const double* coords12, int k, double* A40) {
  if (k == 0) {
    p1_to_p2_tet_divt_tet_cell_integral_0_otherwise f;
    f.tabulate_tensor(A40, nullptr, coords12, 0);
  } else if (k == 1) {
    p1_to_p2_tet_divt_tet_cell_integral_1_otherwise f;
    f.tabulate_tensor(A40, nullptr, coords12, 0);
  } else {
    p1_to_p2_tet_divt_tet_cell_integral_2_otherwise f;
    f.tabulate_tensor(A40, nullptr, coords12, 0);
  }
}

// P2 Laplace element matrix of the reference's FEniCS form (10 x 10, UFC local node order).
void ref_p2_tet_diffusion(const double* coords12, double* K100) {
  p2_tet_diffusion_cell_integral_0_otherwise f;
  f.tabulate_tensor(K100, nullptr, coords12, 0);
}

}  // extern "C"
