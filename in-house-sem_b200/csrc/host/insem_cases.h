/*
 * insem_cases.h -- native case setup of the standalone B200 backend.
 *
 * Turns a model description (macro mesh, discretisation, materials,
 * boundaries, sources, receivers, time settings) into the packed per-step
 * arrays of include/insem_cuda.h, following the reference's setup path:
 * Simulation::build_forest (cpp/src/sim/simulation.cpp:121-175),
 * DofMap::build (cpp/src/ops/dof_map.cpp:42-260), compute_geometry
 * (cpp/src/geometry/geometry.cpp:44-109) and the Solver constructor's
 * build_domains / build_boundaries / build_coupling / build_sources /
 * build_receivers (cpp/src/solver/solver.cpp:147-568).
 *
 * In a drop-in build the reference's own setup produces these arrays; this
 * library lets the backend build benchmark and serving workloads without the
 * reference.  The stable time step is not computed here: the caller runs the
 * device power iteration (insem_cuda_stable_dt) and sets dt and n_steps.
 */
#ifndef INSEM_CASES_H
#define INSEM_CASES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct insem_case_desc {
  /* macro mesh (mesh::MacroMesh) */
  int32_t quad9;              /* 0: Quad4, 1: Quad9 */
  int32_t axisymmetric;       /* 0: cartesian (x, z), 1: axisymmetric (r, z) */
  int32_t n_nodes;
  const double* nodes;        /* [n_nodes][2] */
  int32_t n_cells;
  const int32_t* cells;       /* [n_cells][4 or 9] */
  const int32_t* cell_region; /* [n_cells] */
  int32_t n_boundary;
  const int32_t* boundary;    /* [n_boundary][3] (cell, face, tag) */
  /* discretisation (Discretization, simulation.hpp:38-48) */
  int32_t order;
  int32_t uniform_level;
  double f_max;
  double points_per_wavelength;
  int32_t max_level;
  int32_t n_regions;
  const double* regions;      /* [n_regions][5] xmin, xmax, zmin, zmax, level */
  int32_t azimuthal_order;
  /* materials by region id (Material, description.hpp) */
  int32_t n_materials;
  const int32_t* material_region;
  const int32_t* material_medium; /* 0 acoustic, 1 elastic */
  const double* material_vp;
  const double* material_vs;
  const double* material_rho;
  /* boundary conditions by tag: 0 free, 1 rigid, 2 absorbing */
  int32_t n_bc;
  const int32_t* bc_tag;
  const int32_t* bc_type;
  /* sources: kind 0 force, 1 moment tensor, 2 monopole, 3 dipole */
  int32_t n_sources;
  const int32_t* source_kind;
  const double* source_position;  /* [n][2] */
  const double* source_components;/* [n][3] */
  const int32_t* stf_kind;        /* insem_cuda_stf_kind */
  const double* stf_params;       /* [n][3] f0, t0, amplitude */
  /* receivers */
  int32_t n_receivers;
  const double* receiver_position;   /* [n][2] */
  const int32_t* receiver_medium;    /* -1 any, 0 acoustic, 1 elastic */
  const int32_t* receiver_qoffsets;  /* [n+1] into receiver_quantities */
  const int32_t* receiver_quantities;/* insem_cuda_quantity */
  /* time */
  int32_t record_every;
  int32_t energy_every;
} insem_case_desc;

/* One output array: key in the flat problem layout ("problem.domains.0.l2g"),
 * dtype 0 float32, 1 float64, 2 int32, 3 uint8. */
typedef struct insem_case_array {
  const char* key;
  int32_t dtype;
  int64_t n;
  const void* data;
} insem_case_array;

typedef struct insem_case_out insem_case_out;

/* Builds the problem; returns 0 or an error code (message in insem_case_last_error). */
int insem_case_build(const insem_case_desc* desc, insem_case_out** out);
int32_t insem_case_n_arrays(const insem_case_out* out);
const insem_case_array* insem_case_array_at(const insem_case_out* out, int32_t i);
void insem_case_free(insem_case_out* out);
const char* insem_case_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* INSEM_CASES_H */
