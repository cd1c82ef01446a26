// runtime.cuh -- host-side objects behind the C-ABI handles.
#pragma once
#include <memory>
#include <string>
#include <vector>

#include "core.cuh"

struct moons_mesh {
  int device = 0;
  cudaStream_t stream = nullptr;
  mg::DGrid dg{};
  std::vector<void*> allocs;   // device allocations owned by the mesh
  std::vector<double> hn[3];   // host copy of node coordinates
  int sn[3] = {0, 0, 0};
  // reduction scratch (deterministic two-level sums)
  double* d_partial = nullptr;   // kRedBlocks * kSlots
  unsigned* d_ticket = nullptr;  // kSlots
  double* d_scal = nullptr;      // kSlots result scalars
  double* h_scal = nullptr;      // pinned host mirror
  static constexpr int kSlots = 16;
  // lifetime: fields, solvers and MHD objects hold a reference, so the mesh
  // outlives them whatever order the caller destroys things in
  int refs = 1;
};

struct moons_sf {
  moons_mesh* m = nullptr;
  mg::DF f{};
  mg::DBC bc{};        // bc.defined == 0 -> field carries no BCs
  int all_neumann = 0;
  bool owns = true;
};

namespace mg {
void mesh_ref(moons_mesh* m);
void mesh_unref(moons_mesh* m);
// launch helpers (enqueue on the mesh stream; no sync)
int launch_del(moons_mesh* m, DF out, DF in, int n, int dir, int pad, int gen);
int launch_pw(moons_mesh* m, int op, DF a, const DF* b, double c);
int launch_bcs(moons_mesh* m, DF u, const DBC& bc, bool implicit);
int launch_plane(moons_mesh* m, DF u, int d, int idx, double v, int mode);
int launch_lap_centered(moons_mesh* m, DF out, DF u, int ghost_zero, int scale_mode, double coeff);
int launch_interp(moons_mesh* m, DF out, DF in, int dir);
// masks driven by the BCs of a field (block_field_extend.f90:232-375)
int mask_ghost_XPeriodic(moons_mesh* m, DF u, const DBC* with);       // with==null: field has no BCs
int mask_ghost_N_XPeriodic(moons_mesh* m, DF u, const DBC* with, int dl_with);
int mask_wall_Dirichlet(moons_mesh* m, DF u, const DBC* with, int dl_with, double v);
int mask_wall_Neumann(moons_mesh* m, DF u, const DBC* with, int dl_with, double v);
int mask_wall_Periodic_single(moons_mesh* m, DF u, const DBC* with, int dl_with, double v);
int ghost_zero_bits(const DBC* with);    // faces whose ghost plane assign_ghost_XPeriodic zeroes
int dirichlet_wall_bits(const DBC* with, int dl);  // faces whose wall plane dot products drop
DF make_df(moons_mesh* m, int dl, double** storage);
int dl_after_diff(int dl, int dir);
}  // namespace mg
