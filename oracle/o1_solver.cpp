// ORACLE — test infrastructure only (checker, never the product path).
//
// O1: a restatement of the reference CPU solver, class Solver in
// src/solver.js:8-516, with JavaScript numerics:
//   - every local is a double (a JS Number);
//   - Float32Array elements (pos, prev, vel, invMass, rho, rhoNear, press,
//     pressNear, dispX/Y/Z, pairD) are rounded to float on every store and
//     read back exactly;
//   - Int32Array / Uint8Array elements hold small integers;
//   - consRest is a plain JS Array, so rest lengths stay double;
//   - hashing is Solver._hash with ToInt32 on double products.
// Loop orders follow the reference line by line (Gauss-Seidel contacts and
// constraints, pair cache for the fluid, descending membership in a cell).
// Built with -ffp-contract=off so no multiply-add is fused.
#include "o1_solver.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "js_numerics.h"

namespace oracle {

static inline float f32(double x) { return (float)x; }

// src/solver.js:9-38
JsSolver::JsSolver(int max_fluid) : maxFluid(max_fluid) {}

// src/solver.js:40-70
void JsSolver::alloc(int n) {
  capacity = n;
  pos.assign(3 * n, 0.f);
  prev.assign(3 * n, 0.f);
  vel.assign(3 * n, 0.f);
  invMass.assign(n, 0.f);
  type.assign(n, 0);
  active.assign(n, 0);
  group.assign(n, 0);
  // cellSize (0.22 in the reference) is a tunable here; the table rule is kept
  tableSize = 1 << (int)std::ceil(std::log2(2.0 * n));
  if (tableSizeOverride > 0) tableSize = tableSizeOverride;
  cellStart.assign(tableSize + 1, 0);
  cellEntries.assign(n, 0);
  fluidNext = 0;
  maxPairs = maxFluid * 32;
  pairI.assign(maxPairs, 0);
  pairJ.assign(maxPairs, 0);
  pairD.assign(maxPairs, 0.f);
  pairCount = 0;
  rho.assign(n, 0.f);
  rhoNear.assign(n, 0.f);
  press.assign(n, 0.f);
  pressNear.assign(n, 0.f);
  dispX.assign(n, 0.f);
  dispY.assign(n, 0.f);
  dispZ.assign(n, 0.f);
  nbrCnt.assign(n, 0);
}

// src/solver.js:72-123
void JsSolver::addSolidCube(double cx, double cy, double cz, int n, double spacing,
                            double particleMass) {
  alloc(n * n * n + maxFluid);
  const double half = (n - 1) * spacing * 0.5;
  int id = 0;
  for (int ix = 0; ix < n; ix++)
    for (int iy = 0; iy < n; iy++)
      for (int iz = 0; iz < n; iz++) {
        const int i3 = id * 3;
        pos[i3] = f32(cx - half + ix * spacing);
        pos[i3 + 1] = f32(cy - half + iy * spacing);
        pos[i3 + 2] = f32(cz - half + iz * spacing);
        invMass[id] = f32(1 / particleMass);
        type[id] = SOLID;
        active[id] = 1;
        group[id] = 0;
        id++;
      }
  solidCount = id;

  consA.clear();
  consB.clear();
  consRest.clear();
  consAlive.clear();
  pairSet.clear();
  auto idx = [n](int ix, int iy, int iz) { return (ix * n + iy) * n + iz; };
  const double maxD2 = 3 * spacing * spacing + 1e-6;
  for (int ix = 0; ix < n; ix++)
    for (int iy = 0; iy < n; iy++)
      for (int iz = 0; iz < n; iz++)
        for (int dx = -1; dx <= 1; dx++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dz = -1; dz <= 1; dz++) {
              const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
              if (jx < 0 || jy < 0 || jz < 0 || jx >= n || jy >= n || jz >= n) continue;
              const int a = idx(ix, iy, iz), b = idx(jx, jy, jz);
              if (b <= a) continue;
              const double d2 = (double)(dx * dx + dy * dy + dz * dz) * spacing * spacing;
              if (d2 > maxD2) continue;
              consA.push_back(a);
              consB.push_back(b);
              consRest.push_back(std::sqrt(d2));
              consAlive.push_back(1);
              pairSet.insert((int64_t)a * capacity + b);
            }
  snapPos.assign(pos.begin(), pos.begin() + solidCount * 3);
  snapRest = consRest;
}

// src/solver.js:125-137
void JsSolver::resetSolid() {
  std::copy(snapPos.begin(), snapPos.end(), pos.begin());
  std::copy(snapPos.begin(), snapPos.end(), prev.begin());
  std::fill(vel.begin(), vel.begin() + solidCount * 3, 0.f);
  consRest = snapRest;
  pairSet.clear();
  for (size_t c = 0; c < consA.size(); c++) {
    consAlive[c] = 1;
    pairSet.insert((int64_t)consA[c] * capacity + consB[c]);
  }
  for (int i = 0; i < solidCount; i++) group[i] = 0;
  grabs.clear();
}

// src/solver.js:139-149
void JsSolver::emitFluid(double x, double y, double z, double vx, double vy, double vz,
                         double mass) {
  const int i = solidCount + fluidNext;
  fluidNext = (fluidNext + 1) % maxFluid;
  const int i3 = i * 3;
  pos[i3] = f32(x); pos[i3 + 1] = f32(y); pos[i3 + 2] = f32(z);
  prev[i3] = f32(x); prev[i3 + 1] = f32(y); prev[i3 + 2] = f32(z);
  vel[i3] = f32(vx); vel[i3 + 1] = f32(vy); vel[i3 + 2] = f32(vz);
  invMass[i] = f32(1 / mass);
  type[i] = FLUID;
  active[i] = 1;
}

// src/solver.js:151-159
void JsSolver::clearFluid() { std::fill(active.begin() + solidCount, active.end(), 0); }
int JsSolver::fluidCount() const {
  int m = 0;
  for (int i = solidCount; i < capacity; i++) m += active[i];
  return m;
}

// src/solver.js:162-172
uint32_t JsSolver::hash(double xi, double yi, double zi) const {
  return js_hash(xi, yi, zi, (uint32_t)tableSize);
}
uint32_t JsSolver::hashPos(int i3) const {
  const double inv = 1 / cellSize;
  return hash(std::floor(pos[i3] * inv), std::floor(pos[i3 + 1] * inv),
              std::floor(pos[i3 + 2] * inv));
}

// src/solver.js:174-184
void JsSolver::buildGrid() {
  std::fill(cellStart.begin(), cellStart.end(), 0);
  for (int i = 0; i < capacity; i++)
    if (active[i]) cellStart[hashPos(i * 3)]++;
  int64_t sum = 0;
  for (int k = 0; k < tableSize; k++) {
    sum += cellStart[k];
    cellStart[k] = (int32_t)sum;
  }
  cellStart[tableSize] = (int32_t)sum;
  for (int i = 0; i < capacity; i++)
    if (active[i]) cellEntries[--cellStart[hashPos(i * 3)]] = i;
}

// integrate, src/solver.js:193-202
void JsSolver::passIntegrate(double h) {
  float* p = pos.data(); float* pv = prev.data(); float* v = vel.data();
  for (int i = 0; i < capacity; i++) {
    if (!active[i]) continue;
    const int i3 = i * 3;
    v[i3 + 1] = f32(v[i3 + 1] + gravity * h);
    pv[i3] = p[i3]; pv[i3 + 1] = p[i3 + 1]; pv[i3 + 2] = p[i3 + 2];
    p[i3] = f32(p[i3] + v[i3] * h);
    p[i3 + 1] = f32(p[i3 + 1] + v[i3 + 1] * h);
    p[i3 + 2] = f32(p[i3 + 2] + v[i3 + 2] * h);
  }
}

// mouse grab pull, src/solver.js:204-210
void JsSolver::passGrab() {
  float* p = pos.data();
  for (const Grab& g : grabs) {
    const int i3 = g.i * 3;
    const double k = grabStiffness;
    p[i3] = f32(p[i3] + (g.x - p[i3]) * k);
    p[i3 + 1] = f32(p[i3 + 1] + (g.y - p[i3 + 1]) * k);
    p[i3 + 2] = f32(p[i3 + 2] + (g.z - p[i3 + 2]) * k);
  }
}

// src/solver.js:246-279
void JsSolver::solveContacts() {
  float* p = pos.data();
  const int32_t* cs = cellStart.data();
  const int32_t* ce = cellEntries.data();
  const double inv = 1 / cellSize;
  const double rs = solidRadius, rf = fluidRadius;
  for (int i = 0; i < solidCount; i++) {
    if (!active[i]) continue;
    const int i3 = i * 3;
    const double xi = std::floor(p[i3] * inv), yi = std::floor(p[i3 + 1] * inv),
                 zi = std::floor(p[i3 + 2] * inv);
    const double wi = invMass[i];
    for (int dx = -1; dx <= 1; dx++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dz = -1; dz <= 1; dz++) {
          const uint32_t hsh = hash(xi + dx, yi + dy, zi + dz);
          for (int e = cs[hsh]; e < cs[hsh + 1]; e++) {
            const int j = ce[e];
            if (j <= i || !active[j]) continue;
            const bool solidJ = type[j] == SOLID;
            if (solidJ && pairSet.count((int64_t)i * capacity + j)) continue;
            const int j3 = j * 3;
            const double ddx = (double)p[i3] - p[j3], ddy = (double)p[i3 + 1] - p[j3 + 1],
                         ddz = (double)p[i3 + 2] - p[j3 + 2];
            const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
            const double rsum = rs + (solidJ ? rs : rf);
            if (d2 >= rsum * rsum || d2 < 1e-12) continue;
            const double d = std::sqrt(d2);
            const double wj = invMass[j];
            const double f = (rsum - d) / (d * (wi + wj));
            p[i3] = f32(p[i3] + ddx * f * wi);
            p[i3 + 1] = f32(p[i3 + 1] + ddy * f * wi);
            p[i3 + 2] = f32(p[i3 + 2] + ddz * f * wi);
            p[j3] = f32(p[j3] - ddx * f * wj);
            p[j3 + 1] = f32(p[j3 + 1] - ddy * f * wj);
            p[j3 + 2] = f32(p[j3 + 2] - ddz * f * wj);
          }
        }
  }
}

// src/solver.js:284-354
void JsSolver::solveFluid() {
  float* p = pos.data();
  const int32_t* cs = cellStart.data();
  const int32_t* ce = cellEntries.data();
  const double inv = 1 / cellSize;
  const double H = fluidH, H2 = H * H;
  const double maxPair = 0.05 * H;
  const double maxTotal = 0.35 * H;

  std::fill(rho.begin() + solidCount, rho.end(), 0.f);
  std::fill(rhoNear.begin() + solidCount, rhoNear.end(), 0.f);
  int np = 0;
  for (int i = solidCount; i < capacity; i++) {
    if (!active[i]) continue;
    const int i3 = i * 3;
    const double xi = std::floor(p[i3] * inv), yi = std::floor(p[i3 + 1] * inv),
                 zi = std::floor(p[i3 + 2] * inv);
    for (int dx = -1; dx <= 1; dx++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dz = -1; dz <= 1; dz++) {
          const uint32_t hsh = hash(xi + dx, yi + dy, zi + dz);
          for (int e = cs[hsh]; e < cs[hsh + 1]; e++) {
            const int j = ce[e];
            if (j <= i || !active[j] || type[j] != FLUID) continue;
            const int j3 = j * 3;
            const double ddx = (double)p[j3] - p[i3], ddy = (double)p[j3 + 1] - p[i3 + 1],
                         ddz = (double)p[j3 + 2] - p[i3 + 2];
            const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
            if (d2 >= H2 || np >= maxPairs) continue;
            const double d = std::sqrt(d2);
            const double q = 1 - d / H;
            pairI[np] = i; pairJ[np] = j; pairD[np] = f32(d); np++;
            const double q2 = q * q;
            rho[i] = f32(rho[i] + q2); rho[j] = f32(rho[j] + q2);
            rhoNear[i] = f32(rhoNear[i] + q2 * q); rhoNear[j] = f32(rhoNear[j] + q2 * q);
          }
        }
  }
  pairCount = np;

  for (int i = solidCount; i < capacity; i++) {
    press[i] = f32(stiffness * (rho[i] - restDensity));
    pressNear[i] = f32(nearStiffness * rhoNear[i]);
    dispX[i] = 0; dispY[i] = 0; dispZ[i] = 0;
  }

  for (int k = 0; k < np; k++) {
    const int i = pairI[k], j = pairJ[k];
    const double d = pairD[k];
    if (d < 1e-9) continue;
    const double q = 1 - d / H;
    double D = 0.25 * (((double)press[i] + press[j]) * q +
                       ((double)pressNear[i] + pressNear[j]) * q * q);
    if (D > maxPair) D = maxPair;
    else if (D < -maxPair) D = -maxPair;
    const int i3 = i * 3, j3 = j * 3;
    const double f = D / d;
    const double ddx = ((double)p[j3] - p[i3]) * f, ddy = ((double)p[j3 + 1] - p[i3 + 1]) * f,
                 ddz = ((double)p[j3 + 2] - p[i3 + 2]) * f;
    dispX[i] = f32(dispX[i] - ddx); dispY[i] = f32(dispY[i] - ddy); dispZ[i] = f32(dispZ[i] - ddz);
    dispX[j] = f32(dispX[j] + ddx); dispY[j] = f32(dispY[j] + ddy); dispZ[j] = f32(dispZ[j] + ddz);
  }

  for (int i = solidCount; i < capacity; i++) {
    if (!active[i]) continue;
    double sx = dispX[i], sy = dispY[i], sz = dispZ[i];
    const double s2 = sx * sx + sy * sy + sz * sz;
    if (s2 > maxTotal * maxTotal) {
      const double f = maxTotal / std::sqrt(s2);
      sx *= f; sy *= f; sz *= f;
    }
    const int i3 = i * 3;
    p[i3] = f32(p[i3] + sx); p[i3 + 1] = f32(p[i3 + 1] + sy); p[i3 + 2] = f32(p[i3 + 2] + sz);
  }
}

// src/solver.js:356-381
void JsSolver::solveConstraints(double h) {
  float* p = pos.data();
  const double alpha = compliance / (h * h);
  for (size_t c = 0; c < consA.size(); c++) {
    if (!consAlive[c]) continue;
    const int a = consA[c], b = consB[c];
    const int a3 = a * 3, b3 = b * 3;
    const double wa = invMass[a], wb = invMass[b];
    const double w = wa + wb;
    if (w == 0) continue;
    const double dx = (double)p[a3] - p[b3], dy = (double)p[a3 + 1] - p[b3 + 1],
                 dz = (double)p[a3 + 2] - p[b3 + 2];
    const double d = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (d < 1e-9) continue;
    const double rest = consRest[c];
    if (d > rest * breakStrain) {
      killConstraint((int)c);
      continue;
    }
    const double C = d - rest;
    const double dl = -C / (w + alpha);
    const double f = dl / d;
    p[a3] = f32(p[a3] + dx * f * wa); p[a3 + 1] = f32(p[a3 + 1] + dy * f * wa);
    p[a3 + 2] = f32(p[a3 + 2] + dz * f * wa);
    p[b3] = f32(p[b3] - dx * f * wb); p[b3 + 1] = f32(p[b3 + 1] - dy * f * wb);
    p[b3 + 2] = f32(p[b3 + 2] - dz * f * wb);
    const double strain = C / rest;
    if (std::fabs(strain) > plasticThreshold) consRest[c] += C * plasticRate;
  }
}

// src/solver.js:383-387
void JsSolver::killConstraint(int c) {
  consAlive[c] = 0;
  pairSet.erase((int64_t)consA[c] * capacity + consB[c]);
  componentsDirty = true;
}

// src/solver.js:389-427
void JsSolver::solveBounds() {
  float* p = pos.data();
  const float* pv = prev.data();
  for (int i = 0; i < capacity; i++) {
    if (!active[i]) continue;
    const int i3 = i * 3;
    const bool solid = type[i] == SOLID;
    const double r = solid ? solidRadius : fluidRadius;
    if (p[i3 + 1] < r) {
      p[i3 + 1] = f32(r);
      const double mu = solid ? floorFrictionSolid : floorFrictionFluid;
      p[i3] = f32(p[i3] - ((double)p[i3] - pv[i3]) * mu);
      p[i3 + 2] = f32(p[i3 + 2] - ((double)p[i3 + 2] - pv[i3 + 2]) * mu);
    }
    if (p[i3 + 1] < wallHeight + r) {
      const double lim = r + wallHalfThick;
      for (int ax : {0, 2}) {
        const double wpos = ax == 0 ? wallX : wallZ;
        const double q = p[i3 + ax];
        if (std::fabs(std::fabs(q) - wpos) < lim) {
          const double side = js_sign_or1(q);
          const bool inside = std::fabs(q) < wpos;
          p[i3 + ax] = f32(inside ? side * (wpos - lim) : side * (wpos + lim));
        }
      }
    }
    if (!solid) {
      const double dx = p[i3], dz = p[i3 + 2];
      if (p[i3 + 1] < -3 || dx * dx + dz * dz > cullRadius * cullRadius) active[i] = 0;
    }
  }
}

// velocity update + damping, src/solver.js:218-234
void JsSolver::passVelocity(double h) {
  float* p = pos.data(); float* pv = prev.data(); float* v = vel.data();
  const double invH = 1 / h;
  const double dampS = js_max0(1 - solidDamping * h);
  const double dampF = js_max0(1 - fluidDamping * h);
  for (int i = 0; i < capacity; i++) {
    if (!active[i]) continue;
    const int i3 = i * 3;
    v[i3] = f32(((double)p[i3] - pv[i3]) * invH);
    v[i3 + 1] = f32(((double)p[i3 + 1] - pv[i3 + 1]) * invH);
    v[i3 + 2] = f32(((double)p[i3 + 2] - pv[i3 + 2]) * invH);
    const double damp = type[i] == SOLID ? dampS : dampF;
    v[i3] = f32(v[i3] * damp); v[i3 + 1] = f32(v[i3 + 1] * damp); v[i3 + 2] = f32(v[i3 + 2] * damp);
    const double sp2 = (double)v[i3] * v[i3] + (double)v[i3 + 1] * v[i3 + 1] +
                       (double)v[i3 + 2] * v[i3 + 2];
    if (sp2 > maxSpeed * maxSpeed) {
      const double f = maxSpeed / std::sqrt(sp2);
      v[i3] = f32(v[i3] * f); v[i3 + 1] = f32(v[i3 + 1] * f); v[i3 + 2] = f32(v[i3 + 2] * f);
    }
  }
}

// src/solver.js:431-454
void JsSolver::applyViscosity() {
  float* v = vel.data();
  const double k = viscosity;
  std::fill(dispX.begin() + solidCount, dispX.end(), 0.f);
  std::fill(dispY.begin() + solidCount, dispY.end(), 0.f);
  std::fill(dispZ.begin() + solidCount, dispZ.end(), 0.f);
  std::fill(nbrCnt.begin() + solidCount, nbrCnt.end(), 0);
  for (int q = 0; q < pairCount; q++) {
    const int i = pairI[q], j = pairJ[q];
    const int i3 = i * 3, j3 = j * 3;
    dispX[i] = f32(dispX[i] + v[j3]); dispY[i] = f32(dispY[i] + v[j3 + 1]);
    dispZ[i] = f32(dispZ[i] + v[j3 + 2]); nbrCnt[i]++;
    dispX[j] = f32(dispX[j] + v[i3]); dispY[j] = f32(dispY[j] + v[i3 + 1]);
    dispZ[j] = f32(dispZ[j] + v[i3 + 2]); nbrCnt[j]++;
  }
  for (int i = solidCount; i < capacity; i++) {
    const int m = nbrCnt[i];
    if (!m || !active[i]) continue;
    const int i3 = i * 3;
    v[i3] = f32(v[i3] + k * ((double)dispX[i] / m - v[i3]));
    v[i3 + 1] = f32(v[i3 + 1] + k * ((double)dispY[i] / m - v[i3 + 1]));
    v[i3 + 2] = f32(v[i3 + 2] + k * ((double)dispZ[i] / m - v[i3 + 2]));
  }
}

// src/solver.js:187-242
void JsSolver::step(double dt, int substeps) {
  const double h = dt / substeps;
  for (int s = 0; s < substeps; s++) {
    passIntegrate(h);
    passGrab();
    buildGrid();
    solveContacts();
    solveFluid();
    solveConstraints(h);
    solveBounds();
    passVelocity(h);
    applyViscosity();
  }
  if (componentsDirty) {
    recomputeGroups();
    componentsDirty = false;
  }
}

// src/solver.js:458-486
int JsSolver::cut(double ox, double oy, double oz, double d1x, double d1y, double d1z,
                  double d2x, double d2y, double d2z) {
  const double nx = d1y * d2z - d1z * d2y;
  const double ny = d1z * d2x - d1x * d2z;
  const double nz = d1x * d2y - d1y * d2x;
  const double nLen = std::sqrt(nx * nx + ny * ny + nz * nz);
  if (nLen < 1e-8) return 0;
  const float* p = pos.data();
  int cuts = 0;
  for (size_t c = 0; c < consA.size(); c++) {
    if (!consAlive[c]) continue;
    const int a3 = consA[c] * 3, b3 = consB[c] * 3;
    const double sa = (p[a3] - ox) * nx + (p[a3 + 1] - oy) * ny + (p[a3 + 2] - oz) * nz;
    const double sb = (p[b3] - ox) * nx + (p[b3 + 1] - oy) * ny + (p[b3 + 2] - oz) * nz;
    if (sa * sb >= 0) continue;
    const double t = sa / (sa - sb);
    const double px = p[a3] + ((double)p[b3] - p[a3]) * t - ox;
    const double py = p[a3 + 1] + ((double)p[b3 + 1] - p[a3 + 1]) * t - oy;
    const double pz = p[a3 + 2] + ((double)p[b3 + 2] - p[a3 + 2]) * t - oz;
    const double c1 = (d1y * pz - d1z * py) * nx + (d1z * px - d1x * pz) * ny +
                      (d1x * py - d1y * px) * nz;
    const double c2 = (py * d2z - pz * d2y) * nx + (pz * d2x - px * d2z) * ny +
                      (px * d2y - py * d2x) * nz;
    if (c1 < 0 || c2 < 0) continue;
    killConstraint((int)c);
    cuts++;
  }
  return cuts;
}

// src/solver.js:488-499
void JsSolver::recomputeGroups() {
  const int n = solidCount;
  std::vector<int32_t> parent(n);
  for (int i = 0; i < n; i++) parent[i] = i;
  auto find = [&parent](int x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  for (size_t c = 0; c < consA.size(); c++) {
    if (!consAlive[c]) continue;
    const int ra = find(consA[c]), rb = find(consB[c]);
    if (ra != rb) parent[ra] = rb;
  }
  for (int i = 0; i < n; i++) group[i] = find(i);
}

// src/solver.js:502-515
int JsSolver::pickSolid(double ox, double oy, double oz, double dx, double dy, double dz,
                        double maxPerp, double* tOut) const {
  const float* p = pos.data();
  int best = -1;
  double bestT = INFINITY;
  for (int i = 0; i < solidCount; i++) {
    const int i3 = i * 3;
    const double px = p[i3] - ox, py = p[i3 + 1] - oy, pz = p[i3 + 2] - oz;
    const double t = px * dx + py * dy + pz * dz;
    if (t < 0 || t >= bestT) continue;
    const double qx = px - dx * t, qy = py - dy * t, qz = pz - dz * t;
    if (qx * qx + qy * qy + qz * qz > maxPerp * maxPerp) continue;
    best = i;
    bestT = t;
  }
  if (tOut) *tOut = bestT;
  return best;
}

}  // namespace oracle
