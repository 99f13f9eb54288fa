/* Oracle end-to-end flows -- TEST INFRASTRUCTURE ONLY (see prism_oracle.h). */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "prism_oracle.h"

void or_autotune_f32(const float* data, const or_geom* g, double eb, double rel_eb,
                     const or_intp* in, float errors[18]);
void or_autotune_f64(const double* data, const or_geom* g, double eb, double rel_eb,
                     const or_intp* in, double errors[18]);

#define T float
#define FN(x) x##_f32
#include "pipeline_impl.h"
#undef T
#undef FN
#define T double
#define FN(x) x##_f64
#include "pipeline_impl.h"
#undef T
#undef FN
