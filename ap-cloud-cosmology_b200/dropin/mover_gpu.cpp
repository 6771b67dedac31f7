/*
 * The reference's Mover (mover.h) with its bodies on libapcloud_gpu.so: the octree build,
 * the computational-particle selection, the interpolation and the kick / drift run on the
 * B200 through the C ABI.  Compiled against the reference's own mover.h, it replaces
 * mover.cpp (and with it octree.cpp) in the reference's build; Controller::solve
 * (controller.cpp:54-241) is unchanged.
 *
 * Reference behaviour kept:
 *   - select_computational_particles returns nc + nv + nb, or -1 when the temp-node budget
 *     (maxnc doubling up to 1,000,000, mover.cpp:17-49) is exceeded;
 *   - move_velocity / move_position return the reference's maximum velocity / position
 *     change (mover.cpp:51-121) and update the caller's Physical_particle arrays;
 *   - the Computational_particle vectors are filled after each selection
 *     (octree.cpp:2720-3000), so code that reads them (the adaptive time step,
 *     controller.cpp:146-164; the viewer) sees the reference's cells.
 * A failing library call prints its message and returns the reference's error value
 * instead of exit()ing.
 */
#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

#include "apc_dropin.h"
#include "mover.h"

namespace {
std::mutex g_mu;
std::map<const Computational_particle *, apc_dropin_entry> g_entries;
int g_precision = APC_PREC_FP64;
long g_kicks = 0;

bool ok(apc_context *ctx, int rc, const char *where) {
  if (rc == APC_OK) return true;
  std::fprintf(stderr, "%s: %s (%s)\n", where, apc_status_string(rc), ctx ? apc_last_error(ctx) : "");
  return false;
}
}  // namespace

apc_dropin_entry *apc_dropin_lookup(const Computational_particle *cp) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_entries.find(cp);
  if (it == g_entries.end()) it = g_entries.emplace(cp, apc_dropin_entry{nullptr, 0, nullptr}).first;
  return &it->second;
}

void apc_dropin_release(const Computational_particle *cp) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = g_entries.find(cp);
  if (it == g_entries.end()) return;
  if (it->second.ctx) apc_destroy(it->second.ctx);
  g_entries.erase(it);
}

extern "C" void apc_dropin_set_precision(int precision) { g_precision = precision; }
extern "C" long apc_dropin_kicks(void) { return g_kicks; }
extern "C" void apc_dropin_reset_kicks(void) { g_kicks = 0; }

Mover::Mover(Physical_particle *physical_particle1, Computational_particle *computational_particle1)
    : physical_particle(physical_particle1), computational_particle(computational_particle1) {
  octree = nullptr;  // the octree lives on the GPU
  maxnc = 10000;
}

Mover::~Mover() { apc_dropin_release(computational_particle); }

int Mover::select_computational_particles() {
  apc_dropin_entry *e = apc_dropin_lookup(computational_particle);
  Physical_particle *p = physical_particle;
  if (!e->ctx) {
    apc_config c;
    apc_config_default(&c);
    c.n_particles = p->size;
    c.depth = Octree_Depth;
    c.bc = BC;
    c.box[0] = x_min;
    c.box[1] = x_max;
    c.box[2] = y_min;
    c.box[3] = y_max;
    c.box[4] = z_min;
    c.box[5] = z_max;
    c.gfd_c = GFD_Constant;
    c.maxnc = maxnc;
    c.nmax_cap = 1000000;  // MAXNC of mover.cpp:20
    c.precision = g_precision;
    if (e->argc > 0 &&
        !ok(nullptr, apc_config_from_options(&c, e->argc, (const char *const *)e->argv), "apc_config_from_options"))
      return -1;
    if (!ok(nullptr, apc_create(&c, &e->ctx), "apc_create")) return -1;
  }
  apc_context *ctx = e->ctx;
  // the host arrays are the particle state the caller owns: take them as they are now
  if (!ok(ctx, apc_set_particles(ctx, p->x, p->y, p->z, p->v_x, p->v_y, p->v_z), "apc_set_particles")) return -1;
  int m = -1;
  const int rc = apc_select(ctx, &m);
  if (rc == APC_ERR_NMAX) {
    std::printf("Not enough memory for computational particles.\n");  // mover.cpp:41
    return -1;
  }
  if (!ok(ctx, rc, "apc_select")) return -1;
  int nc = 0, nv = 0, nb = 0, nn = 0;
  if (!ok(ctx, apc_get_cell_counts(ctx, &nc, &nv, &nb, &nn), "apc_get_cell_counts")) return -1;
  Computational_particle *cp = computational_particle;
  const int M = nc + nv;
  cp->size = M;
  cp->nc = nc;
  cp->nv = nv;
  cp->nb = nb;
  cp->x.resize(M);
  cp->y.resize(M);
  cp->z.resize(M);
  cp->CellLength.resize(M);
  cp->IndexOfFirstPhysicalParticle.resize(M);
  cp->NumberOfPhysicalParticles.resize(M);
  cp->Type.resize(M);
  cp->FirstNeigh.resize(M);
  cp->NumberNeigh.resize(M);
  cp->Neigh24.resize(nn);
  for (std::vector<double> *v : {&cp->Density, &cp->Potential, &cp->p_x, &cp->p_y, &cp->p_z, &cp->p_xx, &cp->p_yy,
                                 &cp->p_zz, &cp->p_xy, &cp->p_xz, &cp->p_yz})
    v->assign(M, 0.0);
  if (!ok(ctx,
          apc_get_cells(ctx, cp->x.data(), cp->y.data(), cp->z.data(), cp->CellLength.data(),
                        cp->IndexOfFirstPhysicalParticle.data(), cp->NumberOfPhysicalParticles.data(), cp->Type.data(),
                        cp->FirstNeigh.data(), cp->NumberNeigh.data(), cp->Neigh24.data()),
          "apc_get_cells"))
    return -1;
  return m;
}

double Mover::move_velocity(double dt) {
  apc_dropin_entry *e = apc_dropin_lookup(computational_particle);
  double dv = 0.0;
  if (!ok(e->ctx, e->ctx ? apc_move_velocity(e->ctx, dt, Constant_For_Mover_Velocity, &dv) : APC_ERR_ORDER,
          "apc_move_velocity"))
    return -1.0;
  ++g_kicks;
  return dv;
}

double Mover::move_position(double dt) {
  apc_dropin_entry *e = apc_dropin_lookup(computational_particle);
  double dx = 0.0;
  if (!ok(e->ctx, e->ctx ? apc_move_position(e->ctx, dt, Constant_For_Mover_Position, &dx) : APC_ERR_ORDER,
          "apc_move_position"))
    return -1.0;
  Physical_particle *p = physical_particle;
  if (!ok(e->ctx, apc_get_particles(e->ctx, p->x, p->y, p->z, p->v_x, p->v_y, p->v_z, p->a_x, p->a_y, p->a_z),
          "apc_get_particles"))
    return -1.0;
  return dx;
}
