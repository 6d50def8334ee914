// ORACLE — test infrastructure only (checker, never the product path).
//
// O2: a restatement of the reference's GPU kernels (src/gpu/wgsl.js) run in
// the pass order of GpuSim.encode (src/gpu/sim.js:333-398), templated on the
// arithmetic type R (float = the per-pass FP32 oracle, double = the FP64
// re-run used for drift). Each kernel body is evaluated one invocation at a
// time in index order; gather kernels only write their own slot, so the
// result is independent of invocation order.
//
// Deliberate conventions (shared with the CUDA product, which is checked
// against this file):
//   1. Hash-cell coordinates are Math.floor(p * (1/cellSize)) in double, the
//      convention of Solver._hashPos (src/solver.js:166-172), instead of the
//      WGSL f32 floor(p / cellSize) (src/gpu/wgsl.js:116-118); hashing is
//      Solver._hash with ToInt32 (src/solver.js:162-164). Grids then agree
//      bit for bit with the CPU solver.
//   2. Bucket membership is deterministic: descending particle index inside
//      a bucket, as Solver._buildGrid leaves it (src/solver.js:182-183); the
//      WGSL atomic-cursor scatter (src/gpu/wgsl.js:238-245) has no fixed order.
//   3. The wedge cut and the pick follow Solver.cut / Solver.pickSolid in
//      double precision (src/solver.js:458-486, 502-515).
//   4. Extra rule switches of the CPU solver (tear_mode, plastic_clamp,
//      contact_scale) default to the WGSL rules.
// Floating-point expressions keep the WGSL operand order; the oracle is
// compiled with -ffp-contract=off.
#pragma once
#include <cstdint>
#include <deque>
#include <vector>

#include "../include/upbd.h"

namespace oracle {

template <class R> struct V3 { R x, y, z; };
template <class R> struct V4 { R x, y, z, w; };
template <class R> struct V2 { R x, y; };

template <class R> struct O2Params {
  R h, gravity, solidRadius, fluidRadius, cellSize, fluidH, restDensity, stiffness;
  R nearStiffness, viscosity, compliance, omega, plasticThreshold, plasticRate, tearGap, maxSpeed;
  R wallX, wallZ, wallH, wallT, cullR, dampSolid, dampFluid, frictionSolid;
  R frictionFluid, grabK, sleepSpeed, spacing, solidViscosity, breakStrain, contactScale;
  double invCell;
  int tearMode, plasticClamp;
};

template <class R> struct O2Sim {
  // sizes (src/gpu/sim.js:83-89)
  int S = 0, N1 = 0, dim1 = 0, dim2 = 0, F = 0, N = 0, C = 0, NT = 0, T = 0;
  int substeps = 5, iters = 3;
  uint32_t features = 0;
  upbd_scene_desc desc{};
  upbd_params prm{};
  O2Params<R> P{};
  // state
  std::vector<V4<R>> pos, prev, vel, delta;
  std::vector<V2<R>> density;
  std::vector<uint32_t> flags;
  std::vector<uint32_t> consA, consB, consAlive;
  std::vector<R> consRest;
  std::vector<uint32_t> adj;  // [S+1 offsets][2C ids]
  std::vector<uint32_t> tetIdx;  // 4 per tet
  std::vector<R> tetVol;         // rest volume (negative = dead)
  std::vector<uint32_t> tetAdj;  // [S+1 offsets][4NT ids]
  std::vector<uint32_t> ccount, clist;  // solid contact cache
  // grid
  std::vector<uint32_t> counts, start, entries;
  // initial state for reset
  std::vector<V4<R>> initPos;
  std::vector<R> initRest, initTetVol;
  // frame bookkeeping
  int fluidNext = 0, frames = 0;
  struct Emit { int count, start; V4<R> pos, dir, side, up; } emit{};
  bool emitPending = false;
  struct Cut { double o[3], d1[3], d2[3]; };
  std::deque<Cut> cuts;
  double grabDelta[3] = {0, 0, 0};  // per-frame accumulated mouse motion (JS Numbers)
  V3<R> grabDeltaSub{0, 0, 0};      // per-substep share (f32 uniform)
  uint32_t grabLattice = 0xffff;
  V4<R> grabC{0, 0, 0, 0};
  uint32_t healthBits = 0;

  int create(const upbd_scene_desc& d, const upbd_params& p);
  void setParams(const upbd_params& p);
  void resetSolid();
  void drain();
  uint32_t activeCount() const;

  // passes (pass ids of upbd.h)
  uint32_t cellHashOf(const V4<R>& p, int dx, int dy, int dz) const;
  void passEmit();
  void passIntegrate();
  void passGrid();
  void passDensity();
  void passDisp();
  void passApplyFluid();
  void passCollectContacts();
  void passSolidSolve();
  void passApplySolid();
  void passSolveTets();
  void passSolidContacts();
  void passApplySolidContacts();
  void passBondUpdate();
  void passTetUpdate();
  void passContacts();
  void passApplyAll();
  void passBounds();
  void passVelocity();
  void passSolidVisc();
  void passSolidViscApply();
  void passXsph();
  void passXsphApply();
  uint32_t passCut(const Cut& c);
  void passCutTets(const Cut& c);
  R latticeRest(uint32_t a, uint32_t b) const;
  bool latticeAdjacent(uint32_t i, uint32_t j) const;
  bool isBonded(uint32_t i, uint32_t j) const;
  R solidRsum(uint32_t i, uint32_t j) const;

  void substep(R h, int lastPass = 1000);
  void step(double dt, int nsub);
  void stepH(double h, int nsub);
  void frame();
  int pick(const double ro[3], const double rd[3], double maxPerp, double* t) const;
  void grabSelect(const float c[3], float radius, uint32_t lattice);
  void grabIndices(const uint32_t* idx, int n, const float* w, const float* t3);
  void release();
  void emitParticles(int n, const float* p3, const float* v3, double mass);
  void groups(int32_t* out) const;
};

}  // namespace oracle
