// batch.cuh — device-side description of many independent solves advanced
// together (pulse sweeps, served requests).
//
// Every instance keeps its own tables and state in HBM (same plane layout as
// the single-solve path: upper-triangle planes [e][k]). A class of instances
// with the same band count N shares one tile table: a tile is KT consecutive
// k points of one instance. Stage and observable kernels are persistent: a
// fixed grid walks the tile table, so the table can change between chunks
// without touching the captured CUDA graph.
//
// Time: each instance carries a host-built field table (field at t and
// t + dt/2 for every step, plus t itself), so the device never evaluates the
// laser and the values are the ones the single-solve path uses. The step
// counter of an instance is double buffered by tick parity: kernels of tick
// T read it[T & 1], the observable kernel of tick T writes it[(T + 1) & 1].
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../../include/edus_b200.h"
#include "dev.cuh"

namespace edus {
namespace batch {

// Most k-gradient neighbours of a batch instance (hexagonal and square grids use 12).
constexpr int kBatchMaxNb = 24;

// Field table row of one step: t, E(t) = {pump x,y,z, 0.5 probe x,y,z}, E(t + dt/2).
struct FieldRow {
  double t;
  double pad;
  double Et[6];
  double Eh[6];
  double pad2[2];
};
static_assert(sizeof(FieldRow) == 128, "field rows are 128 bytes");

struct Inst {
  int n, ntri, nk, nnb;
  int n1, n2, lattice, pad1;   // grid k = i1 * n2 + i2; lattice: stencil given by off[]
  int nch, nbands, itfi, res;
  int want_current, want_tabs, ntiles, pad0;
  double dt, wx2, scaleJ, scaleTA;
  double dt6, dt3;         // dt / 6 and dt / 3 of the RK4 stage updates (IEEE divisions, once on the host)
  const int* nbr;          // [nnb][nk]
  const void* H;           // [ntri][nk]   double2 (FP64) or float2 (mixed)
  const void* D;           // [3][ntri][nk]
  const void* GE;          // [3][ntri][nk] or null
  const void* U;           // [n*n][nk]
  // FP64: P0 = rho, Pa / Pb = RK4 stage inputs. Mixed precision: P0 = rho - rho_eq
  // (FP64), Pa / Pb hold FP32 deviations (float2 at the same plane index).
  double2 *P0, *P1, *Pa, *Pb;
  const double2* Peq;      // mixed precision: rho_eq, the initial state [ntri][nk]
  const double* Hdiag;     // mixed precision: diagonal of H in FP64 [n][nk]
  const void* W;           // mixed precision: E-linear rho_eq terms [3][ntri][nk] (float2)
  const FieldRow* field;   // [itfi + 2]
  edus_obs* log;           // [itfi / res + 1]
  void* part;              // [ntiles] observable partials
  unsigned int* done;      // arrival counter of the last-tile reduction
  double wb[kMaxNb];
  double bvec[kMaxNb][3];
  int off[kBatchMaxNb][2];   // lattice step (d1, d2) of each b when lattice != 0
  // Terms that are exact zeros for the whole run, skipped by the stage kernels:
  // bit x of fmask is set when field component x (pump or probe) is nonzero at
  // some step (D_x, W_x are read only then); bsel[0..nsel) lists, in b order,
  // the stencil vectors whose gradient coefficient w_b (E_pump . b) can be
  // nonzero (w_b != 0 and b not orthogonal to every pump component in use).
  int fmask, nsel;
  int bsel[kBatchMaxNb];
};

struct Tile {
  int inst;      // slot
  int k0;        // first k point
  int t_in;      // index of the tile within its instance
  int interior;  // lattice stencil: every k + b of the tile's k points is k + (d1 n2 + d2), no wrap
};

// One instance of a class for the observable kernel: its slot, its number of
// observable units (obs_unit(N) consecutive k points each), its last step and
// output resolution.
struct ClassInst {
  int slot, nunits, itfi, res;
};

struct View {
  const Inst* insts;
  int* it[2];            // step counter per slot, by tick parity
  const Tile* tiles;     // tile table of one class
  const int* ntiles;     // its length (device scalar)
  const ClassInst* cinst;  // instance table of the class
  const int* ninst;        // its length (device scalar)
};

// One RK4 stage (0..3, Source_Main/RungeKutta.cpp schedule) over every tile of
// the class; N is the band count, kt the tile length the table was built with,
// occ the register profile (0: 56 registers, more resident warps; 1: more registers).
cudaError_t launch_stage(int N, int kt, int occ, bool mixed, const View& v, int stage, int parity, int grid, cudaStream_t s);
// Observables of the instances due at this tick (it % res == 0) and the
// step-counter advance of every instance of the class (batch_obs.cu);
// max_inst bounds the class's instance table.
cudaError_t launch_obs(int N, int kt, bool mixed, const View& v, int parity, int max_inst, int grid, cudaStream_t s);
// Persistent grid sizes (SMs x resident blocks) of the two kernels.
int stage_grid(int N, int kt, int occ, bool mixed);
int obs_grid(int N, bool mixed, int max_inst);
bool class_supported(int N, int kt);
// Matrix-product form of the stage kernel (batch_mm.cu), register profile 2 (FP64 batches).
bool mm_supported(int N, int kt);
cudaError_t launch_stage_mm(int N, int kt, bool mixed, const View& v, int stage, int parity, int grid, cudaStream_t s);
int stage_grid_mm(int N, int kt, bool mixed);
// Mixed-precision stage kernel with asynchronous staging (batch_pipe.cu) for
// lattice-stencil instances: register profile 3 (element-parallel
// commutator, cb = 0) and 4 (commutator from register blocks of C = P H~^T,
// cb = 1). Classes it is built for, launch and persistent grid; nsel / ncomp
// are the most stencil vectors and field components in use by an instance of
// the class (they size the staging).
bool pipe_supported(int N, int kt, int cb);
cudaError_t launch_stage_pipe(int N, int kt, int cb, const View& v, int stage, int parity, int nsel, int ncomp, int grid,
                              cudaStream_t s);
int stage_grid_pipe(int N, int kt, int cb, int nsel, int ncomp);
size_t obs_part_bytes();
// k points per observable unit (one partial per unit; the partials are sized per tile)
int obs_unit(int N);
// Mixed precision: W of one instance (after its D and rho_eq are on the device).
cudaError_t launch_weq(const Inst* insts, int slot, int ntri, int nk, cudaStream_t s);

}  // namespace batch
}  // namespace edus
