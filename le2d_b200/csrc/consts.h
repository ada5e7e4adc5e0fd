// Step constants of a sweep, derived from the task's dt, spacing and material
// exactly as the reference derives its Courant numbers (in `real`,
// simple/le_core.c:468-469 and :511-512); the derived factors of the face-form
// update are rounded once from double.  Shared by the single-solve path and the
// batched engine so that both compute identical step constants.
#pragma once

#include "le_core.h"
#include "le2d_kernels.h"

namespace le2d {

inline Sweep<real> make_sweep(real dt, const le_material& m, real h) {
  const real k1 = dt * m.c1 / h;
  const real k2 = dt * m.c2 / h;
  Sweep<real> s;
  s.irhoc1 = m.irhoc1;
  s.irhoc2 = m.irhoc2;
  s.kc1 = (real)((1.0 - (double)k1) / 2.0);
  s.kc2 = (real)((1.0 - (double)k2) / 2.0);
  s.hk1 = (real)(0.5 * (double)k1);
  s.hk2 = (real)(0.5 * (double)k2);
  s.hk1rc1 = (real)(0.5 * (double)k1 * (double)m.rhoc1);
  s.hk1rc3 = (real)(0.5 * (double)k1 * (double)m.rhoc3);
  s.hk2rc2 = (real)(0.5 * (double)k2 * (double)m.rhoc2);
  s.k1 = k1;
  s.k2 = k2;
  s.rhoc1 = m.rhoc1;
  s.rhoc2 = m.rhoc2;
  s.rhoc3 = m.rhoc3;
  s.irp.x = s.irhoc1;
  s.irp.y = s.irhoc2;
  s.nirp.x = -s.irhoc1;
  s.nirp.y = -s.irhoc2;
  s.kcp.x = s.kc1;
  s.kcp.y = s.kc2;
  s.nkcp.x = -s.kc1;
  s.nkcp.y = -s.kc2;
  return s;
}

inline StepConsts<real> make_consts(real dt, const le_vec2& h, const le_material& m) {
  StepConsts<real> c;
  c.x = make_sweep(dt, m, h.x);
  c.y = make_sweep(dt, m, h.y);
  return c;
}

// Rows padded to 128 bytes.
inline long long row_pitch_elems(int nx) {
  const int align = 128 / (int)sizeof(real);
  return ((long long)nx + align - 1) / align * align;
}

}  // namespace le2d
