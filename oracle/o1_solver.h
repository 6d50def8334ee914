// ORACLE — test infrastructure only (checker, never the product path).
// O1: restatement of class Solver, src/solver.js:8-516. See o1_solver.cpp.
#pragma once
#include <cstdint>
#include <unordered_set>
#include <vector>

namespace oracle {

struct JsSolver {
  static constexpr uint8_t FLUID = 0, SOLID = 1;  // src/solver.js:5-6

  explicit JsSolver(int max_fluid);

  // tuning, src/solver.js:14-36 (cellSize src/solver.js:50; the fluid
  // damping 0.6 is the constant of src/solver.js:220)
  double gravity = -10.0, solidRadius = 0.09, fluidRadius = 0.075, compliance = 2.5e-4;
  double plasticThreshold = 0.32, plasticRate = 0.04, breakStrain = 2.6;
  double fluidH = 0.19, restDensity = 6.0, stiffness = 0.002, nearStiffness = 0.008;
  double viscosity = 0.3, solidDamping = 1.2, fluidDamping = 0.6;
  double floorFrictionSolid = 0.4, floorFrictionFluid = 0.04;
  double wallX = 3.5, wallZ = 3.5, wallHeight = 0.92, wallHalfThick = 0.07;
  double cullRadius = 7.0, maxSpeed = 14.0, grabStiffness = 0.3, cellSize = 0.22;
  int tableSizeOverride = 0;  // 0 = the reference rule 2^ceil(log2(2n))

  int maxFluid, solidCount = 0, capacity = 0, tableSize = 0, fluidNext = 0;
  int maxPairs = 0, pairCount = 0;
  std::vector<float> pos, prev, vel, invMass;
  std::vector<uint8_t> type, active;
  std::vector<int32_t> group, cellStart, cellEntries;
  std::vector<int32_t> pairI, pairJ, nbrCnt;
  std::vector<float> pairD, rho, rhoNear, press, pressNear, dispX, dispY, dispZ;
  std::vector<int32_t> consA, consB;
  std::vector<double> consRest;
  std::vector<uint8_t> consAlive;
  std::unordered_set<int64_t> pairSet;
  struct Grab { int i; double x, y, z; };
  std::vector<Grab> grabs;
  bool componentsDirty = false;
  std::vector<float> snapPos;
  std::vector<double> snapRest;

  void alloc(int n);
  void addSolidCube(double cx, double cy, double cz, int n, double spacing, double mass);
  void resetSolid();
  void emitFluid(double x, double y, double z, double vx, double vy, double vz, double mass);
  void clearFluid();
  int fluidCount() const;
  uint32_t hash(double xi, double yi, double zi) const;
  uint32_t hashPos(int i3) const;
  void buildGrid();
  void passIntegrate(double h);
  void passGrab();
  void solveContacts();
  void solveFluid();
  void solveConstraints(double h);
  void killConstraint(int c);
  void solveBounds();
  void passVelocity(double h);
  void applyViscosity();
  void step(double dt, int substeps);
  int cut(double ox, double oy, double oz, double d1x, double d1y, double d1z, double d2x,
          double d2y, double d2z);
  void recomputeGroups();
  int pickSolid(double ox, double oy, double oz, double dx, double dy, double dz,
                double maxPerp, double* tOut) const;
};

}  // namespace oracle
