/*
 * cf_oracle_ls.c — CPU oracle of the GN step's acceptance.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only as the checker.
 *
 * Restates, on the host as the reference runs them:
 *   include/fusion_app.h:1352-1375  upload_scaled_delta_x
 *   include/fusion_app.h:1331-1350  correspondence_rmse (records in order)
 *   include/fusion_app.h:427-458    the increment statistics (nodes in order)
 * Norms use the product sums of the device code (fmaf(c, c, fmaf(b, b, a*a)))
 * so that the scaled increment agrees bit for bit.
 */
#include <math.h>
#include <string.h>

#include "../include/cudafusion_b200.h"

#define CFO_EXPORT __attribute__((visibility("default")))

static inline float ls_norm3(float a, float b, float c) { return sqrtf(fmaf(c, c, fmaf(b, b, a * a))); }

CFO_EXPORT void cfo_scale_delta(const float* dx, int N, float max_rot, float max_trans, float scale, float* out) {
  for (int i = 0; i < N; i++) {
    const float* d = dx + 6 * (size_t)i;
    float rn = ls_norm3(d[0], d[1], d[2]), tn = ls_norm3(d[3], d[4], d[5]);
    float rs = 1.0f, ts = 1.0f;
    if (max_rot > 0.0f && rn > max_rot) rs = max_rot / rn;
    if (max_trans > 0.0f && tn > max_trans) ts = max_trans / tn;
    float fr = rs * scale, ft = ts * scale;
    for (int k = 0; k < 3; k++) out[6 * (size_t)i + k] = d[k] * fr;
    for (int k = 3; k < 6; k++) out[6 * (size_t)i + k] = d[k] * ft;
  }
}

/* sums[4] = rn, tn, er, et summed in FP64 in node order; maxima[4]; returns
 * 1 when every rn and tn is finite */
CFO_EXPORT int cfo_update_stats(const float* dx, int N, float update_scale, float max_rot, float max_trans,
                                double* sums, float* maxima) {
  int fin = 1;
  memset(sums, 0, 4 * sizeof(double));
  memset(maxima, 0, 4 * sizeof(float));
  for (int i = 0; i < N; i++) {
    const float* d = dx + 6 * (size_t)i;
    float rn = ls_norm3(d[0], d[1], d[2]), tn = ls_norm3(d[3], d[4], d[5]);
    fin = fin && isfinite(rn) && isfinite(tn);
    float er = update_scale * rn, et = update_scale * tn;
    if (max_rot > 0.0f) er = fminf(er, max_rot);
    if (max_trans > 0.0f) et = fminf(et, max_trans);
    sums[0] += rn; sums[1] += tn; sums[2] += er; sums[3] += et;
    maxima[0] = fmaxf(maxima[0], rn); maxima[1] = fmaxf(maxima[1], tn);
    maxima[2] = fmaxf(maxima[2], er); maxima[3] = fmaxf(maxima[3], et);
  }
  return fin;
}

/* out[0] = sum w r^2, out[1] = sum w over the valid records of positive weight */
CFO_EXPORT void cfo_corr_rmse(const cf_correspondence* c, int M, double* out) {
  double s = 0.0, ws = 0.0;
  for (int i = 0; i < M; i++) {
    if (!c[i].valid || !(c[i].weight > 0.0f)) continue;
    float dx = c[i].src.x - c[i].dst.x, dy = c[i].src.y - c[i].dst.y, dz = c[i].src.z - c[i].dst.z;
    double r = fma((double)c[i].normal.z, (double)dz, fma((double)c[i].normal.y, (double)dy,
                                                           (double)c[i].normal.x * (double)dx));
    double w = (double)fmaxf(0.0f, c[i].weight);
    s = fma(w * r, r, s);
    ws += w;
  }
  out[0] = s;
  out[1] = ws;
}
