/*
 * pf_oracle_sec.c -- CPU restatement of the reference's secondary-particle
 * bookkeeping (src/driver/secondary_particles3d.h:9-467) as
 * SparseSim3DTP::step() uses it (src/driver/sparse_sim3d_tp.cpp:192-337).
 *
 * TEST INFRASTRUCTURE ONLY: the checker the GPU path is compared against;
 * never linked into or called by the product library.
 *
 * Every floating-point expression keeps the reference's operation order.  The
 * one deviation: emitSecondarySpraySeeds3D orders the spray candidates with
 * std::sort by descending score, which leaves equal scores in an unspecified
 * order; here (and on the GPU) equal scores keep ascending particle order.
 * The results agree whenever no two candidates share a score.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pf_oracle.h"

static double dmax(double a, double b) { return a < b ? b : a; } /* std::max(a, b), NaN as it treats it */
static double dmin(double a, double b) { return b < a ? b : a; } /* std::min(a, b) */

static int finite_particle(const double* pos, const double* vel, double vol) {
  return isfinite(pos[0]) && isfinite(pos[1]) && isfinite(pos[2]) && isfinite(vel[0]) && isfinite(vel[1]) &&
         isfinite(vel[2]) && isfinite(vol);
}

static int set_push(pfo_sec_set* s, const double* pos, const double* vel, double vol, int age) {
  if (s->n >= s->cap) return -1;
  memcpy(s->pos + 3 * s->n, pos, 3 * sizeof(double));
  memcpy(s->vel + 3 * s->n, vel, 3 * sizeof(double));
  s->vol[s->n] = vol;
  s->age[s->n] = age;
  ++s->n;
  return 0;
}

/* secondaryVolumeSum3D (:298-305) */
double pfo_sec_volume_sum(const pfo_sec_set* s, double scale) {
  double v = 0.0;
  for (size_t p = 0; p < s->n; ++p) v += s->vol[p] * scale;
  return v;
}

/* advanceSecondarySet3D (:345-427) */
static int advance_set(pfo_sec_set* s, const pfo_sec_domain* d, const pfo_sec_cfg* c, double dt, int type,
                       int lifetime, double accel_y, double drag, pfo_sec_set* reab, pfo_sec_stats* st) {
  if (s->n == 0) return 0;
  const double xlo = d->ox + 0.5 * d->dx, ylo = d->oy + 0.5 * d->dx, zlo = d->oz + 0.5 * d->dx;
  const double xhi = d->ox + ((double)d->nx - 0.5) * d->dx;
  const double yhi = d->oy + ((double)d->ny - 0.5) * d->dx;
  const double zhi = d->oz + ((double)d->nz - 0.5) * d->dx;
  /* secondaryInsideReabsorbBand3D (:318-333) */
  const double margin = dmax(0.0, c->reabsorb_margin_cells) * d->dx;
  const double bx0 = d->ox + (0.5 * d->dx) + margin, by0 = d->oy + (0.5 * d->dx) + margin;
  const double bz0 = d->oz + (0.5 * d->dx) + margin;
  const double bx1 = d->ox + ((double)d->nx - 0.5) * d->dx - margin;
  const double by1 = d->oy + ((double)d->ny - 0.5) * d->dx - margin;
  const double bz1 = d->oz + ((double)d->nz - 0.5) * d->dx - margin;
  const int band = !(bx0 >= bx1 || by0 >= by1 || bz0 >= bz1);
  char* remove = (char*)calloc(s->n + 1, 1);
  for (size_t p = 0; p < s->n; ++p) {
    double* x = s->pos + 3 * p;
    double* v = s->vel + 3 * p;
    if (!finite_particle(x, v, s->vol[p])) {
      st->finite = 0;
      remove[p] = 1;
      if (type == 0) {
        ++st->expired_droplets;
        st->expired_droplet_volume += s->vol[p] * c->particle_volume_scale;
      } else {
        ++st->expired_bubbles;
        st->expired_bubble_volume += s->vol[p] * c->particle_volume_scale;
      }
      continue;
    }
    const int next_age = s->age[p] + 1;
    s->age[p] = next_age;
    if (type == 0) ++st->advected_droplets;
    else ++st->advected_bubbles;
    v[1] += accel_y * dt;
    double damping = dmax(0.0, c->velocity_damping);
    if (drag > 0.0) {
      damping *= exp(-drag * dt);
      if (type == 0) ++st->dragged_droplets;
      else ++st->dragged_bubbles;
    }
    v[0] = v[0] * damping;
    v[1] = v[1] * damping;
    v[2] = v[2] * damping;
    x[0] += v[0] * dt;
    x[1] += v[1] * dt;
    x[2] += v[2] * dt;
    x[0] = dmax(xlo, dmin(xhi, x[0]));
    x[1] = dmax(ylo, dmin(yhi, x[1]));
    x[2] = dmax(zlo, dmin(zhi, x[2]));
    const double volume = s->vol[p] * c->particle_volume_scale;
    const int inside = band && x[0] > bx0 && x[0] < bx1 && x[1] > by0 && x[1] < by1 && x[2] > bz0 && x[2] < bz1;
    if (inside) {
      remove[p] = 1;
      if (reab && set_push(reab, x, v, s->vol[p], 0)) {
        free(remove);
        return -1;
      }
      if (type == 0) {
        ++st->reabsorbed_droplets;
        st->reabsorbed_droplet_volume += volume;
        if (reab) {
          ++st->reabsorbed_droplets_to_primary;
          st->reabsorbed_droplet_volume_to_primary += volume;
        }
      } else {
        ++st->reabsorbed_bubbles;
        st->reabsorbed_bubble_volume += volume;
        if (reab) {
          ++st->reabsorbed_bubbles_to_primary;
          st->reabsorbed_bubble_volume_to_primary += volume;
        }
      }
    } else if (lifetime >= 0 && next_age >= lifetime) {
      remove[p] = 1;
      if (type == 0) {
        ++st->expired_droplets;
        st->expired_droplet_volume += volume;
      } else {
        ++st->expired_bubbles;
        st->expired_bubble_volume += volume;
      }
    }
  }
  /* compactSecondaryParticles3D (:335-343): survivors keep their order */
  size_t w = 0;
  for (size_t r = 0; r < s->n; ++r) {
    if (remove[r]) continue;
    if (w != r) {
      memcpy(s->pos + 3 * w, s->pos + 3 * r, 3 * sizeof(double));
      memcpy(s->vel + 3 * w, s->vel + 3 * r, 3 * sizeof(double));
      s->vol[w] = s->vol[r];
      s->age[w] = s->age[r];
    }
    ++w;
  }
  s->n = w;
  free(remove);
  return 0;
}

/* advanceSecondaryParticles3D (:429-467) */
int pfo_sec_advance(const pfo_sec_domain* d, const pfo_sec_cfg* c, double dt, pfo_sec_set* droplets,
                    pfo_sec_set* bubbles, pfo_sec_set* reab_droplets, pfo_sec_set* reab_bubbles, pfo_sec_stats* st) {
  memset(st, 0, sizeof(*st));
  st->enabled = c->enabled ? 1 : 0;
  st->finite = 1;
  if (c->enabled && dt > 0.0) {
    if (advance_set(droplets, d, c, dt, 0, c->droplet_lifetime_steps, c->gravity * c->droplet_gravity_scale,
                    c->droplet_drag, reab_droplets, st))
      return -1;
    if (advance_set(bubbles, d, c, dt, 1, c->bubble_lifetime_steps, -c->gravity * c->bubble_buoyancy_scale,
                    c->bubble_drag, reab_bubbles, st))
      return -1;
  }
  st->current_droplet_volume = pfo_sec_volume_sum(droplets, c->particle_volume_scale);
  st->current_bubble_volume = pfo_sec_volume_sum(bubbles, c->particle_volume_scale);
  return 0;
}

/* ---- spray emission (emitSecondarySpraySeeds3D, :136-278) --------------- */

typedef struct {
  double pos[3], vel[3], score;
  int impact;
  size_t index;
} cand_t;

static int cand_cmp(const void* pa, const void* pb) {
  const cand_t* a = (const cand_t*)pa;
  const cand_t* b = (const cand_t*)pb;
  if (a->score > b->score) return -1;
  if (a->score < b->score) return 1;
  return a->index < b->index ? -1 : a->index > b->index ? 1 : 0;
}

int pfo_spray_emit(size_t n, const double* pos, const double* vel, const unsigned char* type, const double* vol,
                   const pfo_spray_cfg* c, int frame_index, pfo_sec_set* droplets, pfo_sec_set* bubbles,
                   pfo_spray_stats* st) {
  memset(st, 0, sizeof(*st));
  st->enabled = c->enabled ? 1 : 0;
  st->finite = 1;
  st->requested_particles = c->requested_particles > 0 ? c->requested_particles : 0;
  st->interface_gate_enabled = c->interface_gate ? 1 : 0;
  st->interface_gate_passed = 1;
  st->interface_cells = c->interface_cells;
  st->interface_grad_max = c->interface_grad_max;
  st->interface_curvature_abs_max = c->interface_curvature_abs_max;
  if (!c->enabled || c->requested_particles <= 0) return 0;
  if (c->interface_gate) {
    const int finite_iface = isfinite(c->interface_grad_max) && isfinite(c->interface_curvature_abs_max);
    const int min_cells = c->min_interface_cells > 0 ? c->min_interface_cells : 0;
    const int pass = finite_iface && c->interface_cells >= min_cells &&
                     c->interface_grad_max >= c->min_interface_grad_max &&
                     c->interface_curvature_abs_max >= c->min_interface_curvature_abs_max;
    st->interface_gate_passed = pass ? 1 : 0;
    if (!finite_iface) st->finite = 0;
    if (!pass) return 0;
  }
  /* liquidParticleBounds3D (:128-134) */
  int valid = 0;
  double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
  for (size_t i = 0; i < n; ++i) {
    if (type[i] != 0) continue;
    const double* p = pos + 3 * i;
    if (!valid) {
      memcpy(mn, p, sizeof(mn));
      memcpy(mx, p, sizeof(mx));
      valid = 1;
      continue;
    }
    for (int a = 0; a < 3; ++a) {
      mn[a] = dmin(mn[a], p[a]);
      mx[a] = dmax(mx[a], p[a]);
    }
  }
  if (!valid) return 0;
  const double surface_y = mn[1] + 0.68 * (mx[1] - mn[1]);
  const double impact_y = mn[1] + dmax(0.0, dmin(1.0, c->impact_region_fraction)) * (mx[1] - mn[1]);
  const double cx = 0.5 * (mn[0] + mx[0]);
  const double cz = 0.5 * (mn[2] + mx[2]);
  cand_t* cand = (cand_t*)malloc((n + 1) * sizeof(cand_t));
  size_t nc = 0;
  for (size_t i = 0; i < n; ++i) {
    if (type[i] != 0) continue;
    const double* p = pos + 3 * i;
    const double* v = vel + 3 * i;
    if (!finite_particle(p, v, vol[i])) {
      st->finite = 0;
      continue;
    }
    const double hspeed = sqrt(v[0] * v[0] + v[2] * v[2]);
    const double upward = dmax(0.0, v[1]);
    const double downward = dmax(0.0, -v[1]);
    const double near_surface = dmax(0.0, p[1] - surface_y);
    const int impact = c->impact_splash_candidates && p[1] <= impact_y && downward >= c->impact_downward_speed_min;
    const double lateral = sqrt((p[0] - cx) * (p[0] - cx) + (p[2] - cz) * (p[2] - cz));
    const double depth = dmax(0.0, impact_y - p[1]);
    const double score = near_surface * 4.0 + upward * 2.0 + hspeed * 0.25 + lateral * 0.03 +
                         (impact ? downward * 2.5 + depth * 0.8 : 0.0);
    if (p[1] >= surface_y || upward > 0.02 || hspeed > 0.25 || impact) {
      if (impact) ++st->impact_candidate_liquid_particles;
      cand_t* q = &cand[nc++];
      memcpy(q->pos, p, sizeof(q->pos));
      memcpy(q->vel, v, sizeof(q->vel));
      q->score = score;
      q->impact = impact;
      q->index = i;
    }
  }
  if (nc == 0) {
    for (size_t i = 0; i < n; ++i) {
      if (type[i] != 0 || !finite_particle(pos + 3 * i, vel + 3 * i, vol[i])) continue;
      cand_t* q = &cand[nc++];
      memcpy(q->pos, pos + 3 * i, sizeof(q->pos));
      memcpy(q->vel, vel + 3 * i, sizeof(q->vel));
      q->score = pos[3 * i + 1];
      q->impact = 0;
      q->index = i;
    }
  }
  st->candidate_liquid_particles = (int)nc;
  if (nc == 0) {
    free(cand);
    return 0;
  }
  qsort(cand, nc, sizeof(cand_t), cand_cmp);
  const int requested = c->requested_particles > 0 ? c->requested_particles : 0;
  st->effective_requested_particles = requested;
  const double dfrac = dmax(0.0, dmin(1.0, c->droplet_fraction));
  int ndrop = (int)floor((double)requested * dfrac + 0.5);
  if (ndrop > requested) ndrop = requested;
  if (ndrop < 0) ndrop = 0;
  const int nbub = requested - ndrop > 0 ? requested - ndrop : 0;
  const size_t want = (size_t)(requested * 3 > 1 ? requested * 3 : 1);
  const size_t window = nc < want ? nc : want;
  const double foam_fraction = dmax(0.0, dmin(1.0, c->impact_foam_fraction));
  for (int k = 0; k < ndrop; ++k) {
    const size_t idx = ((size_t)k * 37u + (size_t)frame_index * 11u) % window;
    const cand_t* q = &cand[idx];
    const double dx = q->pos[0] - cx, dz = q->pos[2] - cz;
    const double len = sqrt(dx * dx + dz * dz);
    const double ox = len > 1e-8 ? dx / len : 0.0, oz = len > 1e-8 ? dz / len : 0.0;
    const double lift = 0.18 + 0.035 * (double)((k + frame_index) % 5);
    int foam_stride = requested + 1;
    if (foam_fraction > 0.0) {
      const int f = (int)floor((1.0 / foam_fraction) + 0.5);
      foam_stride = f > 1 ? f : 1;
    }
    const int foam_ready = q->impact && ((k + frame_index) % foam_stride == 0);
    const double np[3] = {q->pos[0] + 0.035 * ox, q->pos[1] + (foam_ready ? 0.025 : 0.04 + 0.01 * (double)(k % 3)),
                          q->pos[2] + 0.035 * oz};
    double nv[3];
    if (foam_ready) {
      nv[0] = 0.08 * ox;
      nv[1] = 0.08;
      nv[2] = 0.08 * oz;
    } else {
      nv[0] = q->vel[0] + 0.16 * ox;
      nv[1] = q->vel[1] + lift;
      nv[2] = q->vel[2] + 0.16 * oz;
    }
    const double speed = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]); /* Vec3::length */
    const int age = foam_ready ? 6 : (speed > 1.0 ? 0 : (k % 4 == 0 ? 5 : 2));
    if (set_push(droplets, np, nv, c->droplet_volume, age)) {
      free(cand);
      return -1;
    }
    if (foam_ready) ++st->foam_ready_droplets;
    ++st->emitted_droplets;
    st->emitted_droplet_volume += c->droplet_volume * c->particle_volume_scale;
  }
  for (int k = 0; k < nbub; ++k) {
    const size_t idx = ((size_t)k * 53u + (size_t)frame_index * 7u) % window;
    const cand_t* q = &cand[idx];
    const double np[3] = {q->pos[0], dmax(mn[1] + 0.25, q->pos[1] - 0.12), q->pos[2]};
    const double nv[3] = {0.0, 0.16, 0.0};
    if (set_push(bubbles, np, nv, c->bubble_volume, 0)) {
      free(cand);
      return -1;
    }
    ++st->emitted_bubbles;
    st->emitted_bubble_volume += c->bubble_volume * c->particle_volume_scale;
  }
  free(cand);
  return 0;
}
