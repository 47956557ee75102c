// Device-side entry of the fixed-profile contraction for the search kernels'
// host code: a Wyckoff search with the cell and profile fixed writes each
// replica's reflection intensities into the contraction session's intensity
// buffer and reads back the chi^2 at each replica's best scale.
#pragma once
#include <cuda_runtime.h>

#include "p6cuda.h"

namespace p6 {
namespace ct {
struct ProfileLink {
  float *intensities;   // max_replicas x n_refl, FP32, row-major
  double *chi2;         // max_replicas: chi^2 at the best scale of the last enqueue
  int n_refl, n_points, max_replicas, device;
};
ProfileLink link(p6_ct_session *s);
// Y = I . P over the first n_active_points points and the fitted-scale chi^2
// of the first n_replicas rows of the intensity buffer, on `stream`.
p6_status enqueue_fitted(p6_ct_session *s, cudaStream_t stream, int n_replicas, int method, int n_active_points);
// The same without the per-replica reduction: the fitted-scale partials
// {a, b} of replica r are part[r * n_parts + t], t < n_parts (summed in
// order t = l, l + 32, ... per lane l, then across the lanes in a fixed
// butterfly, by the caller's kernel).
p6_status enqueue_fitted_partials(p6_ct_session *s, cudaStream_t stream, int n_replicas, int method,
                                  int n_active_points, const double2 **part, int *n_parts);
// sum w y^2 over the first n_active_points points (FP64).
double syy(p6_ct_session *s, int n_active_points);
// Reports (and clears) a tensor-core pipeline wait that ran out.
p6_status check(p6_ct_session *s);
}  // namespace ct
}  // namespace p6
