// Grounded-wire stationary initial field on the GPU (nodal trilinear FEM).
//
// Replaces SolveStationarProblem3d of the reference's CalcStat3D_3T_A
// (MOD/CalcStat3D_3T_A/TaskSP.cpp:1625-2187), direct mode:
//   1. V: sigma-weighted nodal Laplacian with point electrodes -I at A and +I at
//      B of every wire (TaskSP.cpp:1958-1985), penalty 1e30 on boundary nodes;
//   2. A0 = (Ax, Ay, Az): nodal Laplacian / mu0 with right-hand sides
//      -integral(phi_i sigma dV/dc) + the wire's dipoles I * d_c (c = x, y, z),
//      one factorization and 3 * npls solves (TaskSP.cpp:2039-2142).
// Writes v3n.dat (zeros), v3a.dat (V per source) and a0.dat (Ax, Ay, Az per node
// per source) in the reference's binary layout.
#pragma once
#include <array>
#include <string>
#include <vector>

namespace tdem {

struct StationaryTimes {
  double setup_s = 0, factor_gpu_ms = 0, solve_gpu_ms = 0, total_s = 0;
  int n_nodes = 0, n_sources = 0;
  long long nnz_factor = 0;
};

std::string solve_stationary(const std::string& dir, int device, StationaryTimes* times = nullptr);

// Host only (no device): the element and local coordinates {elem, l0, l1, l2} of every
// source point solve_stationary places, in its order (per wire its nSrsRazb dipoles,
// then electrodes A and B).
std::string stationary_source_points(const std::string& dir, std::vector<std::array<double, 4>>& out);

}  // namespace tdem
