// mesher.cpp -- bit-exact reference numbering from a structured voxel scan.
//
// gen_quadmesh_from_phi (mod_gen_quadmesh.f90:22-679) numbers elements in x-fastest scan
// order of the bone voxels, numbers nodes by first appearance over (element, local node),
// colours connected regions by max-label propagation, keeps a region if any of its nodes
// lies on the mesh bounding box (the region of node 1 always), and compacts the element and
// node lists with two quirks: the last element and the last node always survive.
//
// Equivalent formulation used here: elements sharing a node are exactly 26-neighbouring
// bone voxels, so regions are the 26-connected voxel components (union-find); the region
// order of the colour list is the order of the components' first elements; a region touches
// the mesh bounding box iff one of its voxels lies on the bone bounding box.
#include "mesher.h"

#include <algorithm>
#include <cstring>
#include <numeric>

namespace dtc {
namespace {

const signed char kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                   {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
// HEX20 ring order (mod_gen_quadmesh.f90:244-265) on the doubled grid
const signed char kRing[20][3] = {{0, 0, 0}, {1, 0, 0}, {2, 0, 0}, {2, 1, 0}, {2, 2, 0}, {1, 2, 0}, {0, 2, 0},
                                  {0, 1, 0}, {0, 0, 1}, {2, 0, 1}, {2, 2, 1}, {0, 2, 1}, {0, 0, 2}, {1, 0, 2},
                                  {2, 0, 2}, {2, 1, 2}, {2, 2, 2}, {1, 2, 2}, {0, 2, 2}, {0, 1, 2}};

struct UnionFind {
  std::vector<int32_t> p;
  explicit UnionFind(int64_t n) : p(n) { std::iota(p.begin(), p.end(), 0); }
  int32_t find(int32_t a) {
    while (p[a] != a) { p[a] = p[p[a]]; a = p[a]; }
    return a;
  }
  void unite(int32_t a, int32_t b) {
    a = find(a); b = find(b);
    if (a != b) { if (a < b) std::swap(a, b); p[a] = b; }  // root = smaller element index
  }
};

}  // namespace

int64_t gray_value(const dtc_domain_in& in, int64_t v) {
  switch (in.phi_type) {
    case 1: return static_cast<const int8_t*>(in.phi)[v];
    case 2: return static_cast<const int16_t*>(in.phi)[v];
    default: return static_cast<const int32_t*>(in.phi)[v];
  }
}

void grid_coordinate(const dtc_domain_in& in, int nen, int64_t g, double x[3]) {
  const int64_t gx = (nen == 8) ? in.L[0] + 1 : 2 * in.L[0] + 1;
  const int64_t gy = (nen == 8) ? in.L[1] + 1 : 2 * in.L[1] + 1;
  const int64_t iz = g / (gx * gy), iy = (g - iz * gx * gy) / gx, ix = g - iz * gx * gy - iy * gx;
  const int64_t idx[3] = {ix, iy, iz};
  for (int d = 0; d < 3; ++d)
    x[d] = (nen == 8) ? (double)(idx[d] + in.xa_n[d] - 1) * in.delta[d]
                      : ((double)idx[d] / 2.0 + (double)(in.xa_n[d] - 1)) * in.delta[d];
}

bool grid_on_boundary(const int64_t L[3], int nen, int64_t g) {
  const int64_t m = (nen == 8) ? 1 : 2;
  const int64_t gx = m * L[0] + 1, gy = m * L[1] + 1;
  const int64_t iz = g / (gx * gy), iy = (g - iz * gx * gy) / gx, ix = g - iz * gx * gy - iy * gx;
  return ix == 0 || ix == m * L[0] || iy == 0 || iy == m * L[1] || iz == 0 || iz == m * L[2];
}

namespace {

// Bone voxels (gray >= llimit) in x-fastest scan order: their voxel index and coordinates,
// and the element index of every voxel (-1 for none).
template <typename P>
void scan_bone(const P* phi, int64_t llimit, const int64_t L[3], std::vector<int32_t>& elem_of,
               std::vector<int64_t>& evox, std::vector<int32_t>& exyz) {
  int64_t v = 0;
  for (int64_t z = 0; z < L[2]; ++z)
    for (int64_t y = 0; y < L[1]; ++y)
      for (int64_t x = 0; x < L[0]; ++x, ++v)
        if ((int64_t)phi[v] >= llimit) {
          elem_of[v] = (int32_t)evox.size();
          evox.push_back(v);
          exyz.push_back((int32_t)x);
          exyz.push_back((int32_t)y);
          exyz.push_back((int32_t)z);
        }
}

}  // namespace

int plan_mesh(const dtc_domain_in& in, bool numbering, MeshPlan& mp) {
  mp = MeshPlan();
  const int nen = in.elem_type;
  if (nen != 8 && nen != 20) return DTC_ERR_INVALID_ARGUMENT;
  if (!in.phi || (in.phi_type != 1 && in.phi_type != 2 && in.phi_type != 4)) return DTC_ERR_INVALID_ARGUMENT;
  for (int d = 0; d < 3; ++d) if (in.L[d] < 1 || in.L[d] > 4096) return DTC_ERR_INVALID_ARGUMENT;
  mp.nen = nen;
  std::memcpy(mp.L, in.L, sizeof(mp.L));
  const int64_t L0 = in.L[0], L1 = in.L[1], L2 = in.L[2], nvox = L0 * L1 * L2;

  // bone voxels in scan order = element order, with their coordinates
  std::vector<int32_t> elem_of(nvox, -1);
  std::vector<int64_t> evox;
  std::vector<int32_t> exyz;
  evox.reserve(nvox);
  exyz.reserve(3 * nvox);
  switch (in.phi_type) {
    case 1: scan_bone(static_cast<const int8_t*>(in.phi), in.llimit, in.L, elem_of, evox, exyz); break;
    case 2: scan_bone(static_cast<const int16_t*>(in.phi), in.llimit, in.L, elem_of, evox, exyz); break;
    default: scan_bone(static_cast<const int32_t*>(in.phi), in.llimit, in.L, elem_of, evox, exyz); break;
  }
  if (evox.empty()) { mp.status = DTC_DOMAIN_EMPTY; return DTC_OK; }
  const int64_t ne0 = (int64_t)evox.size();

  // node ids by first appearance; a node's boundary flag is known when its id is given
  const int64_t m = (nen == 8) ? 1 : 2;
  const int64_t gx = m * L0 + 1, gy = m * L1 + 1, gz = m * L2 + 1;
  std::vector<int64_t> id_of(gx * gy * gz, 0);
  std::vector<int64_t> grid_of_id(1, -1);   // 1-based
  std::vector<int32_t> first_elem_of_id(1, -1);
  std::vector<uint8_t> bnd_of_id(1, 0);
  const size_t nn_est = (size_t)std::min<int64_t>(gx * gy * gz, (int64_t)nen * ne0) + 1;
  grid_of_id.reserve(nn_est);
  first_elem_of_id.reserve(nn_est);
  bnd_of_id.reserve(nn_est);
  const signed char(*loc)[3] = (nen == 8) ? kCorner : kRing;
  for (int64_t e = 0; e < ne0; ++e) {
    const int64_t vx = exyz[3 * e], vy = exyz[3 * e + 1], vz = exyz[3 * e + 2];
    // the corners at the element's low x face were numbered by its x - 1 neighbour in the row
    const bool run = vx > 0 && elem_of[evox[e] - 1] >= 0;
    for (int a = 0; a < nen; ++a) {
      if (run && loc[a][0] == 0) continue;
      const int64_t ix = m * vx + loc[a][0], iy = m * vy + loc[a][1], iz = m * vz + loc[a][2];
      const int64_t g = ix + gx * (iy + gy * iz);
      if (id_of[g] == 0) {
        id_of[g] = (int64_t)grid_of_id.size();
        grid_of_id.push_back(g);
        first_elem_of_id.push_back((int32_t)e);
        bnd_of_id.push_back(ix == 0 || ix == gx - 1 || iy == 0 || iy == gy - 1 || iz == 0 || iz == gz - 1);
      }
    }
  }
  const int64_t nn0 = (int64_t)grid_of_id.size() - 1;

  // 26-connected components; union-find roots are the components' first elements
  UnionFind uf(ne0);
  int64_t bmin[3] = {L0, L1, L2}, bmax[3] = {-1, -1, -1};
  for (int64_t e = 0; e < ne0; ++e) {
    const int64_t vx = exyz[3 * e], vy = exyz[3 * e + 1], vz = exyz[3 * e + 2];
    const int64_t c[3] = {vx, vy, vz};
    for (int d = 0; d < 3; ++d) { bmin[d] = std::min(bmin[d], c[d]); bmax[d] = std::max(bmax[d], c[d]); }
    int32_t root = (int32_t)e;   // e's root so far (it only joins sets of smaller roots)
    // inside a run along x the neighbours at x - 1 and x are already in the set of the element
    // before: join it, then only the neighbours at x + 1 are new
    const bool run = vx > 0 && elem_of[evox[e] - 1] >= 0;
    if (run) {
      uf.unite(root, (int32_t)e - 1);
      root = uf.find(root);
    }
    for (int dz = -1; dz <= 0; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = run ? 1 : -1; dx <= 1; ++dx) {
          if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) continue;  // only earlier neighbours
          const int64_t x = vx + dx, y = vy + dy, z = vz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= L0 || y >= L1) continue;
          const int32_t o = elem_of[x + L0 * (y + L1 * z)];
          if (o < 0) continue;
          const int32_t ro = uf.find(o);
          if (ro != root) {
            uf.unite(root, ro);
            root = uf.find(root);
          }
        }
  }
  std::vector<int32_t> comp(ne0);
  for (int64_t e = 0; e < ne0; ++e) comp[e] = uf.find((int32_t)e);
  // keep a region if it touches the bone bounding box; the first region always
  std::vector<uint8_t> keep_comp(ne0, 0);
  for (int64_t e = 0; e < ne0; ++e) {
    bool touch = false;
    for (int d = 0; d < 3; ++d) touch = touch || exyz[3 * e + d] == bmin[d] || exyz[3 * e + d] == bmax[d];
    if (touch) keep_comp[comp[e]] = 1;
  }
  keep_comp[comp[0]] = 1;

  // element compaction: kept regions plus, always, the last element
  mp.kept.assign(nvox, 0);
  int64_t ne = 0;
  for (int64_t e = 0; e < ne0; ++e)
    if (keep_comp[comp[e]]) { mp.kept[evox[e]] = 1; ++ne; }
  const int64_t elast = ne0 - 1;
  if (!keep_comp[comp[elast]]) { mp.last_partial = true; ++ne; }
  mp.last_voxel = evox[elast];

  // node compaction: nodes of kept regions plus, always, the last node
  std::vector<int64_t> new_id(nn0 + 1, 0);
  int64_t nn = 0, nb = 0;
  for (int64_t id = 1; id <= nn0; ++id) {
    if (keep_comp[comp[first_elem_of_id[id]]] || id == nn0) {
      new_id[id] = ++nn;
      nb += bnd_of_id[id];
    }
  }
  if (mp.last_partial) {
    mp.last_grid = grid_of_id[nn0];
    mp.last_on_boundary = bnd_of_id[nn0] != 0;
    const int64_t vx = exyz[3 * elast], vy = exyz[3 * elast + 1], vz = exyz[3 * elast + 2];
    for (int a = 0; a < nen; ++a) {
      const int64_t g = (m * vx + loc[a][0]) + gx * ((m * vy + loc[a][1]) + gy * (m * vz + loc[a][2]));
      if (g == mp.last_grid) mp.last_local = a;
    }
  }
  mp.ne = ne; mp.nn = nn; mp.nb = nb;
  mp.n_free_dof = 3 * (nn - nb);
  if (nn == 0 || ne == 0) { mp.status = DTC_DOMAIN_NO_STRUCTURE; return DTC_OK; }
  if (nn < 6) mp.status = DTC_DOMAIN_FEW_NODES;  // the node-count test of :471-473

  if (numbering) {
    mp.elems.reserve(nen * ne);
    for (int64_t e = 0; e < ne0; ++e) {
      if (!keep_comp[comp[e]] && e != elast) continue;
      const int64_t vx = exyz[3 * e], vy = exyz[3 * e + 1], vz = exyz[3 * e + 2];
      for (int a = 0; a < nen; ++a) {
        const int64_t g = (m * vx + loc[a][0]) + gx * ((m * vy + loc[a][1]) + gy * (m * vz + loc[a][2]));
        mp.elems.push_back(new_id[id_of[g]]);
      }
    }
    mp.node_grid.resize(nn);
    for (int64_t id = 1; id <= nn0; ++id)
      if (new_id[id]) mp.node_grid[new_id[id] - 1] = grid_of_id[id];
  }
  return DTC_OK;
}

}  // namespace dtc
