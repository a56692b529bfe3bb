// placeholder entry points (replaced by ss3d_vario.cu and ss3d_cond.cu)
#include "../../include/specsim3d_gpu.h"
extern "C" int ss3d_vario(const double*, const int*, int, int, const int*, const int*, const int*, const int*, double*,
                          int64_t*) { return SS3D_EINVAL; }
extern "C" int ss3d_condition(double*, const int*, int, const double*, const double*, const ss3d_struct*, int, double,
                              const ss3d_cond_params*, const double*, int, int, int, ss3d_cond_stats*, double*, double*,
                              double*, double*, double*, double*, double*) { return SS3D_EINVAL; }
