// mesh_host.h -- host-side integer mesh pipeline (see mesh_host.cpp).
#pragma once

#include <string>
#include <vector>

#include "common.cuh"

namespace mgpu {

struct HostMesh {
  int N = 0, F = 0, nnodes = 0;
  std::vector<double> x;
  std::vector<int> fptr, fnodes, c0, c1, zone;  // 0-based; c1 = -1 on boundary
};

struct HostTopo {
  std::vector<int> cf_ptr, cf, c2c_ptr, c2c;
  std::vector<int> row_ptr, col, diag, cf_slot, mirror;
  std::vector<int> lo_ptr, lo_rows, up_ptr, up_rows;
  int nlev_lo = 0, nlev_up = 0;
};

int load_host_mesh(const MgpuMesh* in, HostMesh& m, std::string& why);
void build_topology(const HostMesh& m, HostTopo& t);
int build_groups(const HostMesh& m, const MgpuCtrl& ctrl, std::vector<DevGroup>& groups, std::vector<int>& fgrp,
                 int& ier, std::string& why);
void rcm_order(const HostMesh& m, std::vector<int>& new_of_old);

}  // namespace mgpu
