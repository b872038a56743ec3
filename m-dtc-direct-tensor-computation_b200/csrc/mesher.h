// mesher.h -- host planner: the reference mesh of one domain, in structured form.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dtc.h"

namespace dtc {

// Result of meshing one domain the way gen_quadmesh_from_phi (mod_gen_quadmesh.f90:22-679)
// does, but kept as per-voxel flags on the structured grid instead of an element list.
struct MeshPlan {
  int32_t status = DTC_DOMAIN_OK;
  int32_t nen = 8;
  int64_t L[3] = {0, 0, 0};
  int64_t ne = 0, nn = 0, nb = 0;   // reference counts (quirk element/node included)
  int64_t n_free_dof = 0;
  std::vector<uint8_t> kept;        // per voxel: element present with its full stiffness
  // The compaction keeps the last element even when its region was dropped; it then keeps
  // only its last node (mod_gen_quadmesh.f90:598-648).  Its stiffness reaches only that
  // node, as the 3x3 block of the element matrix.
  bool last_partial = false;
  int64_t last_voxel = -1;
  int32_t last_local = -1;          // local node index of the kept node in that element
  int64_t last_grid = -1;           // grid index of that node (corner grid / fine grid)
  bool last_on_boundary = false;
  // reference numbering, filled on request
  std::vector<int64_t> elems;       // nen*ne node ids (1-based, 0 = dropped)
  std::vector<int64_t> node_grid;   // nn grid indices of the nodes, in id order
};

int64_t gray_value(const dtc_domain_in& in, int64_t v);

// Returns DTC_OK or DTC_ERR_INVALID_ARGUMENT; per-domain outcome in mp.status.
int plan_mesh(const dtc_domain_in& in, bool numbering, MeshPlan& mp);

// The same for n domains of one element type on the current CUDA device (mesher_dev.cu):
// plans[i] equals plan_mesh's result bit for bit.  stream: a cudaStream_t; the call returns
// when its work on that stream is done.
int mesh_batch_device(const dtc_domain_in* in, int64_t n, MeshPlan* plans, bool numbering, void* stream,
                      std::string& msg);

// Grid geometry helpers: the node grid has (L+1) points per edge for HEX08 and (2L+1) for
// HEX20; coordinates are (g + xa_n - 1)*delta or (g/2 + xa_n - 1)*delta.
void grid_coordinate(const dtc_domain_in& in, int nen, int64_t g, double x[3]);
bool grid_on_boundary(const int64_t L[3], int nen, int64_t g);

}  // namespace dtc
