/* Oracle predictor -- TEST INFRASTRUCTURE ONLY (see prism_oracle.h).
 * Instantiates predictor_impl.h for float and double. */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "prism_oracle.h"

/* Pinned contraction pattern of the reference build, found by comparing the
 * reference's codes and reconstructions with every fused variant. */
or_fp_policy or_policy = {1, 1, 1, 1, 1, 1, 0, -1, -1, -1, -1, -1, -1, -1, -1, 2};
void or_set_policy(const or_fp_policy* p) { or_policy = *p; }
void or_get_policy(or_fp_policy* p) { *p = or_policy; }

void or_intp_default(or_intp* p) { /* parameters.hpp:8-24 */
  p->alpha = 1.75;
  p->beta = 4.0;
  for (int i = 0; i < 4; ++i) { p->use_md[i] = 1; p->use_natural[i] = 0; p->reverse[i] = 0; }
}

double or_alpha(double rel_eb) { /* InterpolationPredictor.cu:2248-2271 */
  const double a1 = 2.0, a2 = 1.75, a3 = 1.5, a4 = 1.25, a5 = 1;
  const double e1 = 1e-1, e2 = 1e-2, e3 = 1e-3, e4 = 1e-4, e5 = 1e-5;
  if (rel_eb >= e1) return a1;
  if (rel_eb >= e2) return a2 + (a1 - a2) * (rel_eb - e2) / (e1 - e2);
  if (rel_eb >= e3) return a3 + (a2 - a3) * (rel_eb - e3) / (e2 - e3);
  if (rel_eb >= e4) return a4 + (a3 - a4) * (rel_eb - e4) / (e3 - e4);
  if (rel_eb >= e5) return a5 + (a4 - a5) * (rel_eb - e5) / (e4 - e5);
  return a5;
}

#define T float
#define FN(x) x##_f32
#define FMA fmaf
#define FABS fabsf
#include "predictor_impl.h"
#undef T
#undef FN
#undef FMA
#undef FABS

#define T double
#define FN(x) x##_f64
#define FMA fma
#define FABS fabs
#include "predictor_impl.h"
#undef T
#undef FN
#undef FMA
#undef FABS
