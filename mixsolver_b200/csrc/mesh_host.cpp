// mesh_host.cpp -- integer mesh pipeline of a case (host side, once per case).
//
// Builds, from the reference's face list, the arrays every kernel indexes:
//   * cell->face lists in ascending face order and the cell->cell lists of
//     build_connectivity (mod_uns_connectivity.f90:28-108), identical arrays;
//   * the cell CSR pattern of build_cell_csr (mod_uns_simple.f90:835-887):
//     self plus unique neighbours, ascending;
//   * face->CSR-slot maps replacing the linear pos_of scans
//     (mod_uns_simple.f90:909-923) of the assembly loops;
//   * the position of each entry's transpose (for the L^T sweep of IC(0));
//   * level sets of the strictly lower / upper triangle for the triangular
//     sweeps and factorisations;
//   * boundary groups (build_bc, mod_uns_bc.f90:155-393) with its error codes;
//   * a reverse Cuthill-McKee cell order (no counterpart in the reference).

#include "mesh_host.h"

#include <algorithm>
#include <cmath>
#include <deque>
#include <numeric>

namespace mgpu {

int load_host_mesh(const MgpuMesh* in, HostMesh& m, std::string& why) {
  if (!in || in->ncells <= 0 || in->nfaces <= 0 || in->nnodes <= 0 || !in->x || !in->fnode_ptr ||
      !in->fnodes || !in->c0 || !in->c1 || !in->zone) {
    why = "mesh: null array or non-positive size";
    return MGPU_E_ARG;
  }
  m.N = in->ncells;
  m.F = in->nfaces;
  m.nnodes = in->nnodes;
  m.x.assign(in->x, in->x + 3 * (long)m.nnodes);
  m.fptr.assign(in->fnode_ptr, in->fnode_ptr + m.F + 1);
  if (m.fptr[0] != 0) {
    why = "mesh: fnode_ptr[0] must be 0";
    return MGPU_E_MESH;
  }
  for (int i = 0; i < m.F; ++i)
    if (m.fptr[i + 1] - m.fptr[i] < 3) {
      why = "mesh: face with fewer than 3 nodes";
      return MGPU_E_MESH;
    }
  const long nfn = m.fptr[m.F];
  m.fnodes.resize(nfn);
  for (long j = 0; j < nfn; ++j) {
    const int v = in->fnodes[j] - 1;
    if (v < 0 || v >= m.nnodes) {
      why = "mesh: invalid node reference";
      return MGPU_E_MESH;
    }
    m.fnodes[j] = v;
  }
  m.c0.resize(m.F);
  m.c1.resize(m.F);
  m.zone.assign(in->zone, in->zone + m.F);
  for (int i = 0; i < m.F; ++i) {
    m.c0[i] = in->c0[i] - 1;
    m.c1[i] = in->c1[i] - 1;
    if (m.c0[i] < 0 || m.c0[i] >= m.N || m.c1[i] < -1 || m.c1[i] >= m.N || m.c1[i] == m.c0[i]) {
      why = "mesh: invalid cell reference";
      return MGPU_E_MESH;
    }
  }
  return 0;
}

void build_topology(const HostMesh& m, HostTopo& t) {
  const int N = m.N, F = m.F;
  // cell -> faces (counting sort in face order)
  t.cf_ptr.assign(N + 1, 0);
  for (int i = 0; i < F; ++i) {
    t.cf_ptr[m.c0[i] + 1]++;
    if (m.c1[i] >= 0) t.cf_ptr[m.c1[i] + 1]++;
  }
  std::partial_sum(t.cf_ptr.begin(), t.cf_ptr.end(), t.cf_ptr.begin());
  t.cf.assign(t.cf_ptr[N], 0);
  std::vector<int> fill(t.cf_ptr.begin(), t.cf_ptr.end() - 1);
  for (int i = 0; i < F; ++i) {
    t.cf[fill[m.c0[i]]++] = i;
    if (m.c1[i] >= 0) t.cf[fill[m.c1[i]]++] = i;
  }
  // cell -> neighbour cells over interior faces, face order
  t.c2c_ptr.assign(N + 1, 0);
  for (int i = 0; i < F; ++i)
    if (m.c1[i] >= 0) {
      t.c2c_ptr[m.c0[i] + 1]++;
      t.c2c_ptr[m.c1[i] + 1]++;
    }
  std::partial_sum(t.c2c_ptr.begin(), t.c2c_ptr.end(), t.c2c_ptr.begin());
  t.c2c.assign(t.c2c_ptr[N], 0);
  fill.assign(t.c2c_ptr.begin(), t.c2c_ptr.end() - 1);
  for (int i = 0; i < F; ++i)
    if (m.c1[i] >= 0) {
      t.c2c[fill[m.c0[i]]++] = m.c1[i];
      t.c2c[fill[m.c1[i]]++] = m.c0[i];
    }
  // CSR pattern: self + unique neighbours, ascending
  t.row_ptr.assign(N + 1, 0);
  t.col.clear();
  t.col.reserve(N + t.c2c.size());
  std::vector<int> row;
  for (int c = 0; c < N; ++c) {
    row.assign(t.c2c.begin() + t.c2c_ptr[c], t.c2c.begin() + t.c2c_ptr[c + 1]);
    row.push_back(c);
    std::sort(row.begin(), row.end());
    row.erase(std::unique(row.begin(), row.end()), row.end());
    t.col.insert(t.col.end(), row.begin(), row.end());
    t.row_ptr[c + 1] = (int)t.col.size();
  }
  const int nnz = (int)t.col.size();
  auto find = [&](int i, int j) {
    auto b = t.col.begin() + t.row_ptr[i], e = t.col.begin() + t.row_ptr[i + 1];
    auto it = std::lower_bound(b, e, j);
    return (it != e && *it == j) ? (int)(it - t.col.begin()) : -1;
  };
  t.diag.resize(N);
  for (int c = 0; c < N; ++c) t.diag[c] = find(c, c);
  t.cf_slot.resize(t.cf.size());
  for (int c = 0; c < N; ++c)
    for (int k = t.cf_ptr[c]; k < t.cf_ptr[c + 1]; ++k) {
      const int f = t.cf[k];
      if (m.c1[f] < 0) {
        t.cf_slot[k] = -1;
        continue;
      }
      const int other = (m.c0[f] == c) ? m.c1[f] : m.c0[f];
      t.cf_slot[k] = find(c, other);
    }
  t.mirror.resize(nnz);
  for (int i = 0; i < N; ++i)
    for (int k = t.row_ptr[i]; k < t.row_ptr[i + 1]; ++k) t.mirror[k] = find(t.col[k], i);
  // level sets
  std::vector<int> lev(N, 0);
  int nlo = 0;
  for (int i = 0; i < N; ++i) {
    int l = 0;
    for (int k = t.row_ptr[i]; k < t.diag[i]; ++k) l = std::max(l, lev[t.col[k]] + 1);
    lev[i] = l;
    nlo = std::max(nlo, l + 1);
  }
  auto bucket = [&](const std::vector<int>& lv, int nl, std::vector<int>& ptr, std::vector<int>& rows) {
    ptr.assign(nl + 1, 0);
    for (int i = 0; i < N; ++i) ptr[lv[i] + 1]++;
    std::partial_sum(ptr.begin(), ptr.end(), ptr.begin());
    rows.assign(N, 0);
    std::vector<int> f2(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < N; ++i) rows[f2[lv[i]]++] = i;
  };
  bucket(lev, nlo, t.lo_ptr, t.lo_rows);
  t.nlev_lo = nlo;
  int nup = 0;
  for (int i = N - 1; i >= 0; --i) {
    int l = 0;
    for (int k = t.diag[i] + 1; k < t.row_ptr[i + 1]; ++k) l = std::max(l, lev[t.col[k]] + 1);
    lev[i] = l;
    nup = std::max(nup, l + 1);
  }
  // rows j > i that row i depends on were assigned above because the loop
  // runs from the last row down
  bucket(lev, nup, t.up_ptr, t.up_rows);
  t.nlev_up = nup;
}

int build_groups(const HostMesh& m, const MgpuCtrl& ctrl, std::vector<DevGroup>& groups, std::vector<int>& fgrp,
                 int& ier, std::string& why) {
  ier = 0;
  if (ctrl.nbc < 0 || ctrl.nbc > MGPU_MAXBC) {
    why = "ctrl: nbc out of range";
    return MGPU_E_ARG;
  }
  double cmax[3] = {-HUGE_VAL, -HUGE_VAL, -HUGE_VAL}, cmin[3] = {HUGE_VAL, HUGE_VAL, HUGE_VAL};
  for (int i = 0; i < m.nnodes; ++i)
    for (int k = 0; k < 3; ++k) {
      cmax[k] = std::max(cmax[k], m.x[3 * i + k]);
      cmin[k] = std::min(cmin[k], m.x[3 * i + k]);
    }
  double crange = 0.0;
  for (int k = 0; k < 3; ++k) crange = std::max(crange, cmax[k] - cmin[k]);
  groups.assign(ctrl.nbc, DevGroup());
  fgrp.assign(m.F, -1);
  for (int i = 0; i < ctrl.nbc; ++i) {
    const MgpuBcSpec& sp = ctrl.bc[i];
    DevGroup& g = groups[i];
    g = DevGroup();
    g.btype = sp.btype;
    for (int k = 0; k < 3; ++k) g.uvel[k] = sp.uvel[k];
    g.pval = sp.pval;
    g.prfl_mean = sp.umean;
    g.prfl_span = sp.uspan;
    g.prfl_origin = sp.uorigin;
    g.prfl_axis = sp.uaxis - 1;
    if (sp.btype == MGPU_BC_VINLET_PARAB && (sp.uspan <= 0.0 || sp.uaxis < 1 || sp.uaxis > 3)) {
      ier = 14;
      why = "velocity-inlet-parabolic needs span > 0 and axis 1|2|3";
      return MGPU_E_BC;
    }
    if (sp.btype == MGPU_BC_MASSINLET) {
      if (ctrl.rho <= 0.0) {
        ier = 13;
        why = "mass-flow-inlet needs rho > 0";
        return MGPU_E_BC;
      }
      g.uspeed = sp.mdot / ctrl.rho;
    }
    if (!ctrl.energy && (sp.ttype != 0 || sp.tval != 0.0 || sp.qval != 0.0)) {
      why = "thermal boundary values need ctrl.energy (the temperature equation)";
      return MGPU_E_ARG;
    }
    g.ttype = sp.ttype;
    g.tval = sp.tval;
    g.qval = sp.qval;
    g.ntbc = 0;
    for (int t = 0; t < ctrl.ntbc && t < MGPU_MAXTBC; ++t) {
      const MgpuTbcPlane& pl = ctrl.tbc[t];
      if (pl.bc != i) continue;
      if (g.ntbc >= 4 || pl.pdir < 1 || pl.pdir > 3) {
        ier = 15;
        why = "tbc_plane: at most 4 planes a zone, direction 1|2|3";
        return MGPU_E_BC;
      }
      g.tbc_pdir[g.ntbc] = pl.pdir - 1;
      g.tbc_pcoord[g.ntbc] = pl.pcoord;
      g.tbc_ttype[g.ntbc] = pl.ttype;
      g.tbc_tval[g.ntbc] = pl.tval;
      g.tbc_qval[g.ntbc] = pl.qval;
      ++g.ntbc;
    }
    g.tbc_tol = g.ntbc > 0 ? 1.0e-4 * crange : 0.0;
    g.has_lid = sp.has_lid ? 1 : 0;
    g.lid_dir = sp.lid_dir - 1;
    if (g.has_lid && (sp.lid_dir < 1 || sp.lid_dir > 3)) {
      why = "lid direction must be 1|2|3";
      return MGPU_E_ARG;
    }
    g.lid_coord = sp.lid_coord;
    for (int k = 0; k < 3; ++k) g.lid_vel[k] = sp.lid_vel[k];
    g.lid_tol = g.has_lid ? 1.0e-4 * crange : 0.0;
    int nb = 0;
    bool known = false;
    for (int k = 0; k < m.F; ++k) {
      if (m.zone[k] == sp.zone) known = true;
      if (m.c1[k] < 0 && m.zone[k] == sp.zone) {
        ++nb;
        fgrp[k] = i;
      }
    }
    if (!known) {
      ier = 10;
      why = "bc refers to unknown zone";
      return MGPU_E_BC;
    }
    if (nb == 0) {
      ier = 11;
      why = "bc zone has no boundary faces";
      return MGPU_E_BC;
    }
  }
  for (int k = 0; k < m.F; ++k)
    if (m.c1[k] < 0 && fgrp[k] < 0) {
      ier = 12;
      why = "boundary face has no bc specification";
      return MGPU_E_BC;
    }
  return 0;
}

// Reverse Cuthill-McKee on the cell graph. Start of each component: the
// unvisited cell of least (degree, index), moved to a pseudo-peripheral cell
// by George-Liu iteration (BFS; restart from the least (degree, index) cell
// of the last level while the eccentricity grows). Neighbours are queued in
// (degree, index) order. The final order is reversed.
void rcm_order(const HostMesh& m, std::vector<int>& new_of_old) {
  HostTopo t;
  build_topology(m, t);
  const int N = m.N;
  std::vector<int> deg(N);
  for (int c = 0; c < N; ++c) deg[c] = t.row_ptr[c + 1] - t.row_ptr[c] - 1;
  auto less = [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; };
  std::vector<char> visited(N, 0);
  std::vector<int> order;
  order.reserve(N);
  std::vector<int> mark(N, -1), levels;
  int stamp = 0;
  // BFS levels from r inside the unvisited component; returns last level
  auto bfs_last = [&](int r, int& ecc, std::vector<int>& last) {
    ++stamp;
    std::vector<int> cur{r}, next;
    mark[r] = stamp;
    ecc = 0;
    while (true) {
      next.clear();
      for (int v : cur)
        for (int k = t.row_ptr[v]; k < t.row_ptr[v + 1]; ++k) {
          const int w = t.col[k];
          if (w == v || visited[w] || mark[w] == stamp) continue;
          mark[w] = stamp;
          next.push_back(w);
        }
      if (next.empty()) break;
      ++ecc;
      cur.swap(next);
    }
    last = cur;
  };
  std::vector<int> cand(N);
  std::iota(cand.begin(), cand.end(), 0);
  std::sort(cand.begin(), cand.end(), less);
  size_t ci = 0;
  std::vector<int> last, nb;
  while ((int)order.size() < N) {
    while (visited[cand[ci]]) ++ci;
    int r = cand[ci], ecc;
    bfs_last(r, ecc, last);
    while (true) {
      int x = *std::min_element(last.begin(), last.end(), less);
      int ex;
      std::vector<int> lx;
      bfs_last(x, ex, lx);
      if (ex > ecc) {
        r = x;
        ecc = ex;
        last.swap(lx);
      } else {
        break;
      }
    }
    std::deque<int> q{r};
    visited[r] = 1;
    while (!q.empty()) {
      const int v = q.front();
      q.pop_front();
      order.push_back(v);
      nb.clear();
      for (int k = t.row_ptr[v]; k < t.row_ptr[v + 1]; ++k) {
        const int w = t.col[k];
        if (w != v && !visited[w]) nb.push_back(w);
      }
      std::sort(nb.begin(), nb.end(), less);
      for (int w : nb) {
        visited[w] = 1;
        q.push_back(w);
      }
    }
  }
  new_of_old.assign(N, 0);
  for (int p = 0; p < N; ++p) new_of_old[order[N - 1 - p]] = p + 1;
}

}  // namespace mgpu
