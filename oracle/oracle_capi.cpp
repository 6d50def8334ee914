// ORACLE — test infrastructure only (checker, never the product path).
// C entry points over O1 (JsSolver) and O2 (O2Sim<float|double>) for the
// ctypes wrapper in oracle/oracle.py.
#include <cstring>
#include <string>

#include "o1_solver.h"
#include "o2_sim.h"

using namespace oracle;

extern "C" {

// ------------------------------------------------------------------ O1
void* o1_create(int max_fluid) { return new JsSolver(max_fluid); }
void o1_destroy(void* h) { delete (JsSolver*)h; }

int o1_set_param(void* h, const char* name, double v) {
  JsSolver& s = *(JsSolver*)h;
  const std::string n(name);
#define P1(field) if (n == #field) { s.field = v; return 0; }
  P1(gravity) P1(solidRadius) P1(fluidRadius) P1(compliance) P1(plasticThreshold)
  P1(plasticRate) P1(breakStrain) P1(fluidH) P1(restDensity) P1(stiffness) P1(nearStiffness)
  P1(viscosity) P1(solidDamping) P1(fluidDamping) P1(floorFrictionSolid) P1(floorFrictionFluid)
  P1(wallX) P1(wallZ) P1(wallHeight) P1(wallHalfThick) P1(cullRadius) P1(maxSpeed)
  P1(grabStiffness) P1(cellSize)
#undef P1
  if (n == "tableSizeOverride") { s.tableSizeOverride = (int)v; return 0; }
  return -1;
}

void o1_add_solid_cube(void* h, double cx, double cy, double cz, int n, double spacing,
                       double mass) {
  ((JsSolver*)h)->addSolidCube(cx, cy, cz, n, spacing, mass);
}

void o1_emit_fluid(void* h, int n, const double* p3, const double* v3, double mass) {
  JsSolver& s = *(JsSolver*)h;
  for (int k = 0; k < n; k++)
    s.emitFluid(p3[3 * k], p3[3 * k + 1], p3[3 * k + 2], v3[3 * k], v3[3 * k + 1], v3[3 * k + 2],
                mass);
}

void o1_sizes(void* h, int* out) {
  JsSolver& s = *(JsSolver*)h;
  out[0] = s.solidCount; out[1] = s.capacity; out[2] = s.tableSize;
  out[3] = (int)s.consA.size(); out[4] = s.maxPairs; out[5] = s.fluidNext; out[6] = s.pairCount;
}

static std::vector<float>* o1_f32(JsSolver& s, const std::string& n) {
  if (n == "pos") return &s.pos;
  if (n == "prev") return &s.prev;
  if (n == "vel") return &s.vel;
  if (n == "invMass") return &s.invMass;
  if (n == "rho") return &s.rho;
  if (n == "rhoNear") return &s.rhoNear;
  if (n == "press") return &s.press;
  if (n == "pressNear") return &s.pressNear;
  if (n == "dispX") return &s.dispX;
  if (n == "dispY") return &s.dispY;
  if (n == "dispZ") return &s.dispZ;
  if (n == "pairD") return &s.pairD;
  return nullptr;
}
static std::vector<int32_t>* o1_i32(JsSolver& s, const std::string& n) {
  if (n == "group") return &s.group;
  if (n == "cellStart") return &s.cellStart;
  if (n == "cellEntries") return &s.cellEntries;
  if (n == "pairI") return &s.pairI;
  if (n == "pairJ") return &s.pairJ;
  if (n == "nbrCnt") return &s.nbrCnt;
  if (n == "consA") return &s.consA;
  if (n == "consB") return &s.consB;
  return nullptr;
}
static std::vector<uint8_t>* o1_u8(JsSolver& s, const std::string& n) {
  if (n == "active") return &s.active;
  if (n == "type") return &s.type;
  if (n == "consAlive") return &s.consAlive;
  return nullptr;
}

long o1_len(void* h, const char* name) {
  JsSolver& s = *(JsSolver*)h;
  if (auto* v = o1_f32(s, name)) return (long)v->size();
  if (auto* v = o1_i32(s, name)) return (long)v->size();
  if (auto* v = o1_u8(s, name)) return (long)v->size();
  if (std::string(name) == "consRest") return (long)s.consRest.size();
  return -1;
}
int o1_get(void* h, const char* name, void* out) {
  JsSolver& s = *(JsSolver*)h;
  if (auto* v = o1_f32(s, name)) { std::memcpy(out, v->data(), v->size() * 4); return 0; }
  if (auto* v = o1_i32(s, name)) { std::memcpy(out, v->data(), v->size() * 4); return 0; }
  if (auto* v = o1_u8(s, name)) { std::memcpy(out, v->data(), v->size()); return 0; }
  if (std::string(name) == "consRest") {
    std::memcpy(out, s.consRest.data(), s.consRest.size() * 8);
    return 0;
  }
  return -1;
}
int o1_set(void* h, const char* name, const void* in) {
  JsSolver& s = *(JsSolver*)h;
  if (auto* v = o1_f32(s, name)) { std::memcpy(v->data(), in, v->size() * 4); return 0; }
  if (auto* v = o1_i32(s, name)) { std::memcpy(v->data(), in, v->size() * 4); return 0; }
  if (auto* v = o1_u8(s, name)) {
    std::memcpy(v->data(), in, v->size());
    if (std::string(name) == "consAlive") {  // keep pairSet consistent
      s.pairSet.clear();
      for (size_t c = 0; c < s.consA.size(); c++)
        if (s.consAlive[c]) s.pairSet.insert((int64_t)s.consA[c] * s.capacity + s.consB[c]);
    }
    return 0;
  }
  if (std::string(name) == "consRest") {
    std::memcpy(s.consRest.data(), in, s.consRest.size() * 8);
    return 0;
  }
  return -1;
}

void o1_step(void* h, double dt, int substeps) { ((JsSolver*)h)->step(dt, substeps); }

// One stage of Solver.step's substep body (src/solver.js:193-236).
int o1_pass(void* hh, int pass, double h) {
  JsSolver& s = *(JsSolver*)hh;
  switch (pass) {
    case 0: s.passIntegrate(h); return 0;
    case 1: s.passGrab(); return 0;
    case 2: s.buildGrid(); return 0;
    case 3: s.solveContacts(); return 0;
    case 4: s.solveFluid(); return 0;
    case 5: s.solveConstraints(h); return 0;
    case 6: s.solveBounds(); return 0;
    case 7: s.passVelocity(h); return 0;
    case 8: s.applyViscosity(); return 0;
    case 9: s.recomputeGroups(); s.componentsDirty = false; return 0;
  }
  return -1;
}

int o1_cut(void* h, const double* o, const double* d1, const double* d2) {
  return ((JsSolver*)h)->cut(o[0], o[1], o[2], d1[0], d1[1], d1[2], d2[0], d2[1], d2[2]);
}
int o1_pick(void* h, const double* o, const double* d, double maxPerp, double* t) {
  return ((JsSolver*)h)->pickSolid(o[0], o[1], o[2], d[0], d[1], d[2], maxPerp, t);
}
void o1_set_grabs(void* h, int n, const int* idx, const double* xyz) {
  JsSolver& s = *(JsSolver*)h;
  s.grabs.clear();
  for (int k = 0; k < n; k++) s.grabs.push_back({idx[k], xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2]});
}
void o1_reset_solid(void* h) { ((JsSolver*)h)->resetSolid(); }
void o1_clear_fluid(void* h) { ((JsSolver*)h)->clearFluid(); }
int o1_fluid_count(void* h) { return ((JsSolver*)h)->fluidCount(); }
int o1_components_dirty(void* h) { return ((JsSolver*)h)->componentsDirty ? 1 : 0; }

// ------------------------------------------------------------------ O2
struct O2H {
  int prec;
  O2Sim<float>* f = nullptr;
  O2Sim<double>* d = nullptr;
};
#define DISPATCH(h, ...) \
  do { O2H* _h = (O2H*)(h); if (_h->prec == 0) { auto& S_ = *_h->f; __VA_ARGS__; } else { auto& S_ = *_h->d; __VA_ARGS__; } } while (0)

void* o2_create(const upbd_scene_desc* desc, const upbd_params* prm, int precision) {
  O2H* h = new O2H{precision};
  int rc;
  if (precision == 0) { h->f = new O2Sim<float>(); rc = h->f->create(*desc, *prm); }
  else { h->d = new O2Sim<double>(); rc = h->d->create(*desc, *prm); }
  if (rc != 0) { delete h->f; delete h->d; delete h; return nullptr; }
  return h;
}
void o2_destroy(void* h) {
  O2H* p = (O2H*)h;
  delete p->f;
  delete p->d;
  delete p;
}
void o2_info(void* h, upbd_info* out) {
  DISPATCH(h, {
    std::memset(out, 0, sizeof(*out));
    out->solid_n = S_.S; out->n1 = S_.N1; out->dim1 = S_.dim1; out->dim2 = S_.dim2;
    out->max_fluid = S_.F; out->total = S_.N; out->num_cons = S_.C; out->num_tets = S_.NT;
    out->table_size = S_.T; out->substeps = S_.substeps; out->solid_iters = S_.iters;
    out->fluid_next = S_.fluidNext; out->features = S_.features; out->frames = S_.frames;
  });
}
void o2_set_params(void* h, const upbd_params* p) { DISPATCH(h, S_.setParams(*p)); }
void o2_step(void* h, double dt, int n) { DISPATCH(h, S_.step(dt, n)); }
void o2_frame(void* h) { DISPATCH(h, S_.frame()); }
void o2_substep_partial(void* h, double hh, int last) {
  DISPATCH(h, { S_.substep((decltype(S_.P.h))hh, last); });
}
void o2_rebuild_grid(void* h) { DISPATCH(h, S_.passGrid()); }
// One pass (UPBD_PASS_* id) on the current state with substep length hh, for
// pass-by-pass comparisons with O1: GRID, DENSITY, DISP (the displacement
// into delta), APPLY_FLUID, CONTACTS (into delta), APPLY_ALL, BOUNDS,
// VELOCITY, XSPH (into delta), XSPH_APPLY. Returns 0, or -1 for another id.
int o2_run_pass(void* h, int pass, double hh) {
  int rc = 0;
  DISPATCH(h, {
    S_.P.h = (decltype(S_.P.h))hh;
    switch (pass) {
      case UPBD_PASS_GRID: S_.passGrid(); break;
      case UPBD_PASS_DENSITY: S_.passDensity(); break;
      case UPBD_PASS_DISP: S_.passDisp(); break;
      case UPBD_PASS_APPLY_FLUID: S_.passApplyFluid(); break;
      case UPBD_PASS_CONTACTS: S_.passContacts(); break;
      case UPBD_PASS_APPLY_ALL: S_.passApplyAll(); break;
      case UPBD_PASS_BOUNDS: S_.passBounds(); break;
      case UPBD_PASS_VELOCITY: S_.passVelocity(); break;
      case UPBD_PASS_XSPH: S_.passXsph(); break;
      case UPBD_PASS_XSPH_APPLY: S_.passXsphApply(); break;
      default: rc = -1;
    }
  });
  return rc;
}
void o2_set_iters(void* h, int iters) { DISPATCH(h, S_.iters = iters); }

// Single passes of the WGSL schedule that o2_run_pass does not cover (ids
// private to the oracle, for the per-pass comparison with the reference's
// kernels run by tests/golden/wgslmini.py).
enum {
  O2X_INTEGRATE = 101, O2X_COLLECT, O2X_SOLID_SOLVE, O2X_APPLY_SOLID, O2X_SOLVE_TETS,
  O2X_APPLY_SOLID_CONTACTS, O2X_SOLID_CONTACTS, O2X_BOND_UPDATE, O2X_TET_UPDATE, O2X_SOLID_VISC,
  O2X_SOLID_VISC_APPLY, O2X_EMIT
};
int o2_run_pass_x(void* h, int pass, double hh, const float* grab_delta_sub) {
  int rc = 0;
  DISPATCH(h, {
    using R = decltype(S_.P.h);
    S_.P.h = (R)hh;
    if (grab_delta_sub) S_.grabDeltaSub = {(R)grab_delta_sub[0], (R)grab_delta_sub[1], (R)grab_delta_sub[2]};
    switch (pass) {
      case O2X_INTEGRATE: S_.passIntegrate(); break;
      case O2X_COLLECT: S_.passCollectContacts(); break;
      case O2X_SOLID_SOLVE: S_.passSolidSolve(); break;
      case O2X_APPLY_SOLID: S_.passApplySolid(); break;
      case O2X_SOLVE_TETS: S_.passSolveTets(); break;
      case O2X_APPLY_SOLID_CONTACTS: S_.passApplySolidContacts(); break;
      case O2X_SOLID_CONTACTS: S_.passSolidContacts(); break;
      case O2X_BOND_UPDATE: S_.passBondUpdate(); break;
      case O2X_TET_UPDATE: S_.passTetUpdate(); break;
      case O2X_SOLID_VISC: S_.passSolidVisc(); break;
      case O2X_SOLID_VISC_APPLY: S_.passSolidViscApply(); break;
      case O2X_EMIT: S_.passEmit(); break;
      default: rc = -1;
    }
  });
  return rc;
}
void o2_write_delta(void* h, const double* d4) {
  DISPATCH(h, {
    using R = decltype(S_.P.h);
    for (int i = 0; i < S_.N; i++) S_.delta[i] = {(R)d4[4*i], (R)d4[4*i+1], (R)d4[4*i+2], (R)d4[4*i+3]};
  });
}
// the solid contact cache: ccount[S] and clist[S * C_K]
void o2_read_contact_cache(void* h, uint32_t* ccount, uint32_t* clist) {
  DISPATCH(h, {
    std::memcpy(ccount, S_.ccount.data(), S_.ccount.size() * 4);
    std::memcpy(clist, S_.clist.data(), S_.clist.size() * 4);
  });
}
void o2_write_contact_cache(void* h, const uint32_t* ccount, const uint32_t* clist) {
  DISPATCH(h, {
    std::memcpy(S_.ccount.data(), ccount, S_.ccount.size() * 4);
    std::memcpy(S_.clist.data(), clist, S_.clist.size() * 4);
  });
}
// tets as the reference packs them: [a, b, c, d, rest volume f32 bits] each
void o2_write_tets(void* h, const uint32_t* tets5) {
  DISPATCH(h, {
    using R = decltype(S_.P.h);
    for (int t = 0; t < S_.NT; t++) {
      for (int q = 0; q < 4; q++) S_.tetIdx[4*t+q] = tets5[5*t+q];
      float v;
      std::memcpy(&v, &tets5[5*t+4], 4);
      S_.tetVol[t] = (R)v;
    }
  });
}

void o2_read_state(void* h, double* pos4, double* prev4, double* vel4, double* dens2,
                   uint32_t* flags) {
  DISPATCH(h, {
    for (int i = 0; i < S_.N; i++) {
      if (pos4) { pos4[4*i] = S_.pos[i].x; pos4[4*i+1] = S_.pos[i].y; pos4[4*i+2] = S_.pos[i].z; pos4[4*i+3] = S_.pos[i].w; }
      if (prev4) { prev4[4*i] = S_.prev[i].x; prev4[4*i+1] = S_.prev[i].y; prev4[4*i+2] = S_.prev[i].z; prev4[4*i+3] = S_.prev[i].w; }
      if (vel4) { vel4[4*i] = S_.vel[i].x; vel4[4*i+1] = S_.vel[i].y; vel4[4*i+2] = S_.vel[i].z; vel4[4*i+3] = S_.vel[i].w; }
      if (dens2) { dens2[2*i] = S_.density[i].x; dens2[2*i+1] = S_.density[i].y; }
      if (flags) flags[i] = S_.flags[i];
    }
  });
}
void o2_write_state(void* h, const double* pos4, const double* prev4, const double* vel4,
                    const double* dens2, const uint32_t* flags) {
  DISPATCH(h, {
    using R = decltype(S_.P.h);
    for (int i = 0; i < S_.N; i++) {
      if (pos4) S_.pos[i] = {(R)pos4[4*i], (R)pos4[4*i+1], (R)pos4[4*i+2], (R)pos4[4*i+3]};
      if (prev4) S_.prev[i] = {(R)prev4[4*i], (R)prev4[4*i+1], (R)prev4[4*i+2], (R)prev4[4*i+3]};
      if (vel4) S_.vel[i] = {(R)vel4[4*i], (R)vel4[4*i+1], (R)vel4[4*i+2], (R)vel4[4*i+3]};
      if (dens2) S_.density[i] = {(R)dens2[2*i], (R)dens2[2*i+1]};
      if (flags) S_.flags[i] = flags[i];
    }
  });
}
void o2_read_delta(void* h, double* d4) {
  DISPATCH(h, {
    for (int i = 0; i < S_.N; i++) {
      d4[4*i] = S_.delta[i].x; d4[4*i+1] = S_.delta[i].y; d4[4*i+2] = S_.delta[i].z; d4[4*i+3] = S_.delta[i].w;
    }
  });
}
void o2_read_constraints(void* h, uint32_t* cons4, double* rest) {
  DISPATCH(h, {
    for (int c = 0; c < S_.C; c++) {
      if (cons4) {
        float r = (float)S_.consRest[c];
        uint32_t bits;
        std::memcpy(&bits, &r, 4);
        cons4[4*c] = S_.consA[c]; cons4[4*c+1] = S_.consB[c]; cons4[4*c+2] = bits;
        cons4[4*c+3] = S_.consAlive[c];
      }
      if (rest) rest[c] = (double)S_.consRest[c];
    }
  });
}
void o2_write_constraints(void* h, const uint32_t* cons4) {
  DISPATCH(h, {
    using R = decltype(S_.P.h);
    for (int c = 0; c < S_.C; c++) {
      float r;
      std::memcpy(&r, &cons4[4*c+2], 4);
      S_.consRest[c] = (R)r;
      S_.consAlive[c] = cons4[4*c+3];
    }
  });
}
void o2_read_adjacency(void* h, uint32_t* adj) {
  DISPATCH(h, std::memcpy(adj, S_.adj.data(), S_.adj.size() * 4));
}
void o2_read_grid(void* h, uint32_t* counts, uint32_t* offsets, uint32_t* entries) {
  DISPATCH(h, {
    if (counts) std::memcpy(counts, S_.counts.data(), S_.counts.size() * 4);
    if (offsets) std::memcpy(offsets, S_.start.data(), S_.start.size() * 4);
    if (entries) std::memcpy(entries, S_.entries.data(), S_.start[S_.T] * 4);
  });
}
void o2_read_tets(void* h, uint32_t* tets5) {
  DISPATCH(h, {
    for (int t = 0; t < S_.NT; t++) {
      for (int q = 0; q < 4; q++) tets5[5*t+q] = S_.tetIdx[4*t+q];
      float v = (float)S_.tetVol[t];
      std::memcpy(&tets5[5*t+4], &v, 4);
    }
  });
}
void o2_read_tet_adjacency(void* h, uint32_t* adj) {
  DISPATCH(h, std::memcpy(adj, S_.tetAdj.data(), S_.tetAdj.size() * 4));
}
void o2_emit(void* h, int count, const float* p, const float* dir, const float* side,
             const float* up, float speed, float phase) {
  DISPATCH(h, {
    using R = decltype(S_.P.h);
    S_.emit.count = count;
    S_.emit.start = S_.fluidNext;
    S_.emit.pos = {(R)p[0], (R)p[1], (R)p[2], (R)speed};
    S_.emit.dir = {(R)dir[0], (R)dir[1], (R)dir[2], (R)phase};
    S_.emit.side = {(R)side[0], (R)side[1], (R)side[2], 0};
    S_.emit.up = {(R)up[0], (R)up[1], (R)up[2], 0};
    S_.emitPending = true;
  });
}
void o2_emit_particles(void* h, int n, const float* p3, const float* v3, double mass) {
  DISPATCH(h, S_.emitParticles(n, p3, v3, mass));
}
uint32_t o2_slice_now(void* h, const double* o, const double* d1, const double* d2) {
  uint32_t n = 0;
  DISPATCH(h, {
    typename std::remove_reference<decltype(S_)>::type::Cut c;
    std::memcpy(c.o, o, 24); std::memcpy(c.d1, d1, 24); std::memcpy(c.d2, d2, 24);
    n = S_.passCut(c);
    if (S_.features & UPBD_FEAT_TETS) S_.passCutTets(c);
  });
  return n;
}
void o2_slice(void* h, const double* o, const double* d1, const double* d2) {
  DISPATCH(h, {
    typename std::remove_reference<decltype(S_)>::type::Cut c;
    std::memcpy(c.o, o, 24); std::memcpy(c.d1, d1, 24); std::memcpy(c.d2, d2, 24);
    S_.cuts.push_back(c);
  });
}
int o2_pick(void* h, const double* ro, const double* rd, double maxPerp, double* t) {
  int id = -1;
  DISPATCH(h, id = S_.pick(ro, rd, maxPerp, t));
  return id;
}
void o2_grab_select(void* h, const float* c, float r, uint32_t lattice) {
  DISPATCH(h, S_.grabSelect(c, r, lattice));
}
void o2_grab_indices(void* h, const uint32_t* idx, int n, const float* w, const float* t3) {
  DISPATCH(h, S_.grabIndices(idx, n, w, t3));
}
void o2_grab_move(void* h, const float* d) {
  DISPATCH(h, { S_.grabDelta[0] += d[0]; S_.grabDelta[1] += d[1]; S_.grabDelta[2] += d[2]; });
}
void o2_release(void* h) { DISPATCH(h, S_.release()); }
void o2_drain(void* h) { DISPATCH(h, S_.drain()); }
uint32_t o2_active_count(void* h) {
  uint32_t n = 0;
  DISPATCH(h, n = S_.activeCount());
  return n;
}
void o2_reset_solid(void* h) { DISPATCH(h, S_.resetSolid()); }
void o2_groups(void* h, int32_t* out) { DISPATCH(h, S_.groups(out)); }
uint32_t o2_health(void* h) {
  uint32_t b = 0;
  DISPATCH(h, b = S_.healthBits);
  return b;
}
int o2_fluid_next(void* h) {
  int n = 0;
  DISPATCH(h, n = S_.fluidNext);
  return n;
}

}  // extern "C"
