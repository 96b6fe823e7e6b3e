/*
 * cf_oracle_impl.h — body of the CPU oracle, instantiated twice by
 * cf_oracle.c: once with R=float (reference operation order, FP32) and once
 * with R=double (the FP64 oracle).  TEST INFRASTRUCTURE ONLY.
 *
 * Every function cites the CUDAFusion source it restates.  Expressions keep
 * the reference's operand order so that the FP32 instantiation reproduces the
 * reference's host-compiled se3 functions bit for bit (see tests/test_oracle_kat.py).
 *
 * Required macros: R (float|double), F(name) (suffixing), SQRT, SIN, COS, EXP,
 * FABS, FMAX.
 */

typedef struct { R x, y, z; } F(v3);
typedef struct { R x, y, z, w; } F(q4);
typedef struct { F(q4) real, dual; } F(dq);
typedef struct { R m[4][4]; } F(m4);

static inline F(v3) F(mk3)(R x, R y, R z) { F(v3) v; v.x = x; v.y = y; v.z = z; return v; }
static inline F(q4) F(mk4)(R x, R y, R z, R w) { F(q4) q; q.x = x; q.y = y; q.z = z; q.w = w; return q; }
static inline F(v3) F(ld3)(cf_vec3 v) { return F(mk3)((R)v.x, (R)v.y, (R)v.z); }
static inline F(dq) F(lddq)(const cf_dual_quat* d) {
  F(dq) r;
  r.real = F(mk4)((R)d->real.x, (R)d->real.y, (R)d->real.z, (R)d->real.w);
  r.dual = F(mk4)((R)d->dual.x, (R)d->dual.y, (R)d->dual.z, (R)d->dual.w);
  return r;
}
static inline void F(stdq)(cf_dual_quat* d, F(dq) r) {
  d->real.x = (float)r.real.x; d->real.y = (float)r.real.y; d->real.z = (float)r.real.z; d->real.w = (float)r.real.w;
  d->dual.x = (float)r.dual.x; d->dual.y = (float)r.dual.y; d->dual.z = (float)r.dual.z; d->dual.w = (float)r.dual.w;
}

static inline F(m4) F(m4_identity)(void) {
  F(m4) T;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) T.m[i][j] = (i == j) ? (R)1 : (R)0;
  return T;
}

/* se3_math.cuh:40-98 — SE(3) exponential with Rodrigues coefficients
 * A = sin t / t, B = (1 - cos t)/t^2, C = (t - sin t)/t^3 and the first-order
 * branch below t = 1e-6. */
static F(m4) F(exp_se3)(const R* tw) {
  R ox = tw[0], oy = tw[1], oz = tw[2];
  R vx = tw[3], vy = tw[4], vz = tw[5];
  R th2 = ox * ox + oy * oy + oz * oz;
  R th = SQRT(th2);
  F(m4) T = F(m4_identity)();
  R A, B, C;
  if (th < (R)1e-6f) {
    A = (R)1; B = (R)0.5f; C = (R)1 / (R)6;
  } else {
    R it = (R)1 / th;
    R it2 = it * it;
    A = SIN(th) * it;
    B = ((R)1 - COS(th)) * it2;
    C = (th - SIN(th)) * it2 * it;
  }
  /* rotation  R = I + A[w]x + B[w]x^2 */
  T.m[0][0] = (R)1 - B * (oy * oy + oz * oz);
  T.m[0][1] = B * ox * oy - A * oz;
  T.m[0][2] = B * ox * oz + A * oy;
  T.m[1][0] = B * ox * oy + A * oz;
  T.m[1][1] = (R)1 - B * (ox * ox + oz * oz);
  T.m[1][2] = B * oy * oz - A * ox;
  T.m[2][0] = B * ox * oz - A * oy;
  T.m[2][1] = B * oy * oz + A * ox;
  T.m[2][2] = (R)1 - B * (ox * ox + oy * oy);
  /* translation t = V v,  V = I + B[w]x + C[w]x^2 */
  R v00 = (R)1 - C * (oy * oy + oz * oz), v01 = C * ox * oy - B * oz, v02 = C * ox * oz + B * oy;
  R v10 = C * ox * oy + B * oz, v11 = (R)1 - C * (ox * ox + oz * oz), v12 = C * oy * oz - B * ox;
  R v20 = C * ox * oz - B * oy, v21 = C * oy * oz + B * ox, v22 = (R)1 - C * (ox * ox + oy * oy);
  T.m[0][3] = v00 * vx + v01 * vy + v02 * vz;
  T.m[1][3] = v10 * vx + v11 * vy + v12 * vz;
  T.m[2][3] = v20 * vx + v21 * vy + v22 * vz;
  return T;
}

/* se3_math.cuh:205-214 — Hamilton product, (x,y,z,w) storage. */
static inline F(q4) F(qmul)(F(q4) a, F(q4) b) {
  return F(mk4)(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
                a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
                a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
static inline F(q4) F(qconj)(F(q4) q) { return F(mk4)(-q.x, -q.y, -q.z, q.w); }
/* se3_math.cuh:223-231 */
static inline F(q4) F(qnormalize)(F(q4) q) {
  R n = SQRT(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  if (n < (R)1e-12f) return F(mk4)(0, 0, 0, 1);
  return F(mk4)(q.x / n, q.y / n, q.z / n, q.w / n);
}
static inline R F(qdot)(F(q4) a, F(q4) b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

static inline F(dq) F(dq_identity)(void) {
  F(dq) d;
  d.real = F(mk4)(0, 0, 0, 1);
  d.dual = F(mk4)(0, 0, 0, 0);
  return d;
}

/* se3_math.cuh:244-300 — rotation matrix to quaternion (four branches keyed
 * on the trace and the largest diagonal entry), then dual = 0.5 * (t,0) * real. */
static F(dq) F(mat4_to_dq)(const F(m4)* T) {
  R tr = T->m[0][0] + T->m[1][1] + T->m[2][2];
  F(q4) q;
  if (tr > 0) {
    R s = SQRT(tr + (R)1) * (R)2;
    q.w = (R)0.25f * s;
    q.x = (T->m[2][1] - T->m[1][2]) / s;
    q.y = (T->m[0][2] - T->m[2][0]) / s;
    q.z = (T->m[1][0] - T->m[0][1]) / s;
  } else if (T->m[0][0] > T->m[1][1] && T->m[0][0] > T->m[2][2]) {
    R s = SQRT((R)1 + T->m[0][0] - T->m[1][1] - T->m[2][2]) * (R)2;
    q.w = (T->m[2][1] - T->m[1][2]) / s;
    q.x = (R)0.25f * s;
    q.y = (T->m[0][1] + T->m[1][0]) / s;
    q.z = (T->m[0][2] + T->m[2][0]) / s;
  } else if (T->m[1][1] > T->m[2][2]) {
    R s = SQRT((R)1 + T->m[1][1] - T->m[0][0] - T->m[2][2]) * (R)2;
    q.w = (T->m[0][2] - T->m[2][0]) / s;
    q.x = (T->m[0][1] + T->m[1][0]) / s;
    q.y = (R)0.25f * s;
    q.z = (T->m[1][2] + T->m[2][1]) / s;
  } else {
    R s = SQRT((R)1 + T->m[2][2] - T->m[0][0] - T->m[1][1]) * (R)2;
    q.w = (T->m[1][0] - T->m[0][1]) / s;
    q.x = (T->m[0][2] + T->m[2][0]) / s;
    q.y = (T->m[1][2] + T->m[2][1]) / s;
    q.z = (R)0.25f * s;
  }
  q = F(qnormalize)(q);
  F(q4) qt = F(mk4)(T->m[0][3], T->m[1][3], T->m[2][3], 0);
  F(q4) qd = F(qmul)(qt, q);
  qd.x *= (R)0.5f; qd.y *= (R)0.5f; qd.z *= (R)0.5f; qd.w *= (R)0.5f;
  F(dq) d;
  d.real = q;
  d.dual = qd;
  return d;
}

/* se3_math.cuh:302-328 */
static F(dq) F(dq_normalize)(F(dq) d) {
  R n = SQRT(d.real.x * d.real.x + d.real.y * d.real.y + d.real.z * d.real.z + d.real.w * d.real.w);
  if (n < (R)1e-12f) return F(dq_identity)();
  R inv = (R)1 / n;
  d.real.x *= inv; d.real.y *= inv; d.real.z *= inv; d.real.w *= inv;
  d.dual.x *= inv; d.dual.y *= inv; d.dual.z *= inv; d.dual.w *= inv;
  return d;
}

/* se3_math.cuh:330-340 */
static F(dq) F(dq_mul)(F(dq) a, F(dq) b) {
  F(dq) r;
  r.real = F(qmul)(a.real, b.real);
  F(q4) u = F(qmul)(a.real, b.dual);
  F(q4) v = F(qmul)(a.dual, b.real);
  r.dual = F(mk4)(u.x + v.x, u.y + v.y, u.z + v.z, u.w + v.w);
  return F(dq_normalize)(r);
}

/* se3_math.cuh:342-347 */
static F(dq) F(dq_from_twist)(const R* tw) {
  F(m4) T = F(exp_se3)(tw);
  return F(mat4_to_dq)(&T);
}

/* se3_math.cuh:349-360 */
static F(v3) F(dq_rotate)(F(dq) d, F(v3) p) {
  F(q4) pq = F(mk4)(p.x, p.y, p.z, 0);
  F(q4) r = F(qmul)(F(qmul)(d.real, pq), F(qconj)(d.real));
  return F(mk3)(r.x, r.y, r.z);
}
/* se3_math.cuh:362-368 */
static F(v3) F(dq_translation)(F(dq) d) {
  F(q4) t = F(qmul)(d.dual, F(qconj)(d.real));
  return F(mk3)((R)2 * t.x, (R)2 * t.y, (R)2 * t.z);
}
/* se3_math.cuh:370-377 */
static F(v3) F(dq_transform_point)(F(dq) d, F(v3) p) {
  F(v3) r = F(dq_rotate)(d, p);
  F(v3) t = F(dq_translation)(d);
  return F(mk3)(r.x + t.x, r.y + t.y, r.z + t.z);
}
/* se3_math.cuh:379-388 */
static F(v3) F(dq_transform_point_centered)(F(dq) d, F(v3) p, F(v3) c) {
  F(v3) rp = F(dq_transform_point)(d, p);
  F(v3) rc = F(dq_rotate)(d, c);
  return F(mk3)(rp.x + c.x - rc.x, rp.y + c.y - rc.y, rp.z + c.z - rc.z);
}
/* se3_math.cuh:390-403 */
static F(dq) F(dq_from_rt)(F(q4) qr, F(v3) t) {
  F(dq) d;
  d.real = F(qnormalize)(qr);
  F(q4) qt = F(mk4)(t.x, t.y, t.z, 0);
  d.dual = F(qmul)(qt, d.real);
  d.dual.x *= (R)0.5f; d.dual.y *= (R)0.5f; d.dual.z *= (R)0.5f; d.dual.w *= (R)0.5f;
  return F(dq_normalize)(d);
}
/* se3_math.cuh:405-415 — node-centred DQ -> plain DQ. */
static F(dq) F(dq_centered)(F(dq) d, F(v3) c) {
  F(v3) t = F(dq_translation)(d);
  F(v3) rc = F(dq_rotate)(d, c);
  F(v3) ct = F(mk3)(t.x + c.x - rc.x, t.y + c.y - rc.y, t.z + c.z - rc.z);
  return F(dq_from_rt)(d.real, ct);
}

/* se3_math.cuh:450-510 (device) / include/fusion_math.h:32-78 (host copy):
 * blend the node-centred DQs of the 4 skinning nodes with the antipodality
 * fix, normalise, transform.  Node ids outside [0, num_nodes) are skipped (the
 * device version reads them unchecked). */
static F(v3) F(warp_point)(F(v3) p, const cf_deform_node* nodes, const cf_dual_quat* T,
                           int num_nodes, const int* ids, const float* ws) {
  F(dq) b;
  b.real = F(mk4)(0, 0, 0, 0);
  b.dual = F(mk4)(0, 0, 0, 0);
  R wsum = 0;
  for (int k = 0; k < CF_K_NEIGHBORS; k++) {
    int nid = ids[k];
    R w = (R)ws[k];
    if (nid < 0 || nid >= num_nodes || w < (R)1e-8f) continue;
    F(dq) d = F(dq_centered)(F(lddq)(&T[nid]), F(ld3)(nodes[nid].pos));
    if (F(qdot)(d.real, b.real) < 0) {
      d.real.x *= -1; d.real.y *= -1; d.real.z *= -1; d.real.w *= -1;
      d.dual.x *= -1; d.dual.y *= -1; d.dual.z *= -1; d.dual.w *= -1;
    }
    b.real.x += w * d.real.x; b.real.y += w * d.real.y; b.real.z += w * d.real.z; b.real.w += w * d.real.w;
    b.dual.x += w * d.dual.x; b.dual.y += w * d.dual.y; b.dual.z += w * d.dual.z; b.dual.w += w * d.dual.w;
    wsum += w;
  }
  if (wsum < (R)1e-8f) return p;
  b = F(dq_normalize)(b);
  return F(dq_transform_point)(b, p);
}

/* src/warp_field.cu:250-291 — clamp, exponentiate, left-compose. */
static F(dq) F(twist_update)(F(dq) T, const float* dx, R max_rot, R max_trans, R scale) {
  R tw[6];
  for (int k = 0; k < 6; k++) tw[k] = scale * (R)dx[k];
  R rn = SQRT(tw[0] * tw[0] + tw[1] * tw[1] + tw[2] * tw[2]);
  if (max_rot > 0 && rn > max_rot) {
    R s = max_rot / rn;
    tw[0] *= s; tw[1] *= s; tw[2] *= s;
  }
  R tn = SQRT(tw[3] * tw[3] + tw[4] * tw[4] + tw[5] * tw[5]);
  if (max_trans > 0 && tn > max_trans) {
    R s = max_trans / tn;
    tw[3] *= s; tw[4] *= s; tw[5] *= s;
  }
  F(dq) dT = F(dq_from_twist)(tw);
  return F(dq_mul)(dT, T);
}

/* kernels/solver_kernels.cu:13-24 */
static inline R F(huber)(R r, R delta) {
  R a = FABS(r);
  return (a <= delta) ? (R)1 : delta / a;
}

/* kernels/solver_kernels.cu:25-44 — binary search of a column in a block row. */
static int F(find_block)(int row, int col, const int* row_ptr, const int* col_idx) {
  int lo = row_ptr[row], hi = row_ptr[row + 1] - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    int v = col_idx[mid];
    if (v == col) return mid;
    if (v < col) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

/* se3_math.cuh:121-145 — point-to-plane Jacobian row of node k. */
static inline void F(jac_row)(F(v3) src, F(v3) x, F(v3) n, R w, R* J) {
  F(v3) l = F(mk3)(src.x - x.x, src.y - x.y, src.z - x.z);
  F(v3) cp = F(mk3)(l.y * n.z - l.z * n.y, l.z * n.x - l.x * n.z, l.x * n.y - l.y * n.x);
  J[0] = w * cp.x; J[1] = w * cp.y; J[2] = w * cp.z;
  J[3] = w * n.x; J[4] = w * n.y; J[5] = w * n.z;
}

/* kernels/solver_kernels.cu:140-165 — 6x3 ARAP Jacobian; row a is d r / d x_a
 * with the reference's sign on the rotation rows (q x e_a), or the consistent
 * sign (e_a x q) when cfo_arap_consistent is set. */
static inline void F(arap_jac)(F(v3) p, R J[6][3]) {
  J[0][0] = 0; J[0][1] = p.z; J[0][2] = -p.y;
  J[1][0] = -p.z; J[1][1] = 0; J[1][2] = p.x;
  J[2][0] = p.y; J[2][1] = -p.x; J[2][2] = 0;
  if (cfo_arap_consistent) /* e_a x q: the true derivative of the left update */
    for (int a = 0; a < 3; a++)
      for (int q = 0; q < 3; q++) J[a][q] = -J[a][q];
  J[3][0] = 1; J[3][1] = 0; J[3][2] = 0;
  J[4][0] = 0; J[4][1] = 1; J[4][2] = 0;
  J[5][0] = 0; J[5][1] = 0; J[5][2] = 1;
}

/* Data term of one correspondence, kernels/solver_kernels.cu:52-138.
 * Accumulates into A (nnzb*36) and b (6N) in R precision; returns the
 * correspondence's energy fw*r^2 (0 when skipped). */
static R F(data_term)(const cf_correspondence* c, F(v3) src, const cf_deform_node* nodes,
                      int N, const int* row_ptr, const int* col_idx, R* A, R* b) {
  if (!c->valid) return 0;
  F(v3) dst = F(ld3)(c->dst), n = F(ld3)(c->normal);
  R res = n.x * (src.x - dst.x) + n.y * (src.y - dst.y) + n.z * (src.z - dst.z);
  R hw = F(huber)(res, (R)0.2f);
  R fw = FMAX((R)c->weight, (R)0) * hw;
  if (fw <= (R)1e-8f) return 0;
  R J[CF_K_NEIGHBORS][6];
  int ok[CF_K_NEIGHBORS] = {0, 0, 0, 0};
  for (int k = 0; k < CF_K_NEIGHBORS; k++) {
    int ni = c->node_ids[k];
    R wi = (R)c->node_ws[k];
    if (ni >= 0 && ni < N && wi > (R)1e-8f) {
      F(jac_row)(src, F(ld3)(nodes[ni].pos), n, wi, J[k]);
      ok[k] = 1;
      for (int a = 0; a < 6; a++) b[ni * 6 + a] += -fw * J[k][a] * res;
    }
  }
  for (int ki = 0; ki < CF_K_NEIGHBORS; ki++) {
    if (!ok[ki]) continue;
    int ni = c->node_ids[ki];
    for (int kj = 0; kj < CF_K_NEIGHBORS; kj++) {
      if (!ok[kj]) continue;
      int nj = c->node_ids[kj];
      int blk = F(find_block)(ni, nj, row_ptr, col_idx);
      if (blk < 0) continue;
      R* B = A + (size_t)blk * 36;
      for (int a = 0; a < 6; a++)
        for (int bb = 0; bb < 6; bb++) B[a * 6 + bb] += fw * J[ki][a] * J[kj][bb];
    }
  }
  return fw * res * res;
}

/* ARAP edges of node ni, kernels/solver_kernels.cu:202-352.  Each undirected
 * pair is visited from its lower-index endpoint, once per occurrence in that
 * endpoint's neighbour list.  Returns the ARAP energy of the visited edges. */
static R F(smooth_term)(int ni, const cf_deform_node* nodes, const cf_dual_quat* T, int N,
                        R lambda, const int* row_ptr, const int* col_idx, R* A, R* b) {
  const cf_deform_node* nd = &nodes[ni];
  R e = 0;
  for (int k = 0; k < nd->num_neighbors && k < CF_K_GRAPH; k++) {
    int nj = nd->neighbors[k];
    if (nj < 0 || nj >= N) continue;
    if (nj <= ni) continue;
    R nw = FMAX((R)nd->neighbor_w[k], (R)0.05f);
    F(v3) xj = F(ld3)(nodes[nj].pos), xi = F(ld3)(nd->pos);
    F(dq) Ti = F(lddq)(&T[ni]), Tj = F(lddq)(&T[nj]);
    F(v3) Ti_xj = F(dq_transform_point_centered)(Ti, xj, xi);
    F(v3) Ti_xi = F(dq_transform_point_centered)(Ti, xi, xi);
    F(v3) Tj_xj = F(dq_transform_point_centered)(Tj, xj, xj);
    F(v3) rest = F(mk3)(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
    F(v3) curr = F(mk3)(Ti_xi.x - Tj_xj.x, Ti_xi.y - Tj_xj.y, Ti_xi.z - Tj_xj.z);
    R dr = SQRT(rest.x * rest.x + rest.y * rest.y + rest.z * rest.z);
    R dc = SQRT(curr.x * curr.x + curr.y * curr.y + curr.z * curr.z);
    R strain = FABS(dc - dr) / FMAX(dr, (R)1e-6f);
    R ratio = strain / (R)0.25f;
    R sw = EXP(-(ratio * ratio));
    F(v3) r = F(mk3)(Ti_xj.x - Tj_xj.x, Ti_xj.y - Tj_xj.y, Ti_xj.z - Tj_xj.z);
    R rn = SQRT(r.x * r.x + r.y * r.y + r.z * r.z);
    R hw = F(huber)(rn, (R)0.05f);
    R el = lambda * nw * hw * sw;
    if (el <= (R)1e-8f) continue;
    e += el * (r.x * r.x + r.y * r.y + r.z * r.z);
    R Ji[6][3], Jj[6][3];
    F(arap_jac)(F(mk3)(Ti_xj.x - xi.x, Ti_xj.y - xi.y, Ti_xj.z - xi.z), Ji);
    F(arap_jac)(F(mk3)(Tj_xj.x - xj.x, Tj_xj.y - xj.y, Tj_xj.z - xj.z), Jj);
    int ii = F(find_block)(ni, ni, row_ptr, col_idx);
    int jj = F(find_block)(nj, nj, row_ptr, col_idx);
    int ij = F(find_block)(ni, nj, row_ptr, col_idx);
    int ji = F(find_block)(nj, ni, row_ptr, col_idx);
    for (int a = 0; a < 6; a++)
      for (int bb = 0; bb < 6; bb++) {
        R vii = 0, vjj = 0, vij = 0, vji = 0;
        for (int q = 0; q < 3; q++) {
          vii += Ji[a][q] * Ji[bb][q];
          vjj += Jj[a][q] * Jj[bb][q];
          vij += Ji[a][q] * Jj[bb][q];
          vji += Jj[a][q] * Ji[bb][q];
        }
        if (ii >= 0) A[(size_t)ii * 36 + a * 6 + bb] += el * vii;
        if (jj >= 0) A[(size_t)jj * 36 + a * 6 + bb] += el * vjj;
        if (ij >= 0) A[(size_t)ij * 36 + a * 6 + bb] += -el * vij;
        if (ji >= 0) A[(size_t)ji * 36 + a * 6 + bb] += -el * vji;
      }
    R rr[3] = {r.x, r.y, r.z};
    for (int a = 0; a < 6; a++) {
      R vi = 0, vj = 0;
      for (int q = 0; q < 3; q++) {
        vi += Ji[a][q] * rr[q];
        vj += Jj[a][q] * rr[q];
      }
      b[ni * 6 + a] += -el * vi;
      b[nj * 6 + a] += el * vj;
    }
  }
  return e;
}

/* kernels/solver_kernels.cu:167-194 — relative Levenberg damping. */
static void F(damping)(int N, const int* row_ptr, const int* col_idx, R lambda, R* A) {
  for (int ni = 0; ni < N; ni++) {
    int blk = F(find_block)(ni, ni, row_ptr, col_idx);
    if (blk < 0) continue;
    R* D = A + (size_t)blk * 36;
    for (int k = 0; k < 6; k++) {
      R d = D[k * 6 + k];
      R fl = (k < 3) ? (R)1e-3f : (R)1e-2f;
      D[k * 6 + k] = d + lambda * FMAX(FABS(d), fl);
    }
  }
}

/* se3_math.cuh:152-202 — 6x6 inverse via Cholesky (lower triangle read). */
static int F(inv6_chol)(const R* A, R* Ainv) {
  R L[6][6];
  memset(L, 0, sizeof(L));
  for (int i = 0; i < 6; i++)
    for (int j = 0; j <= i; j++) {
      R s = A[i * 6 + j];
      for (int k = 0; k < j; k++) s -= L[i][k] * L[j][k];
      if (i == j) {
        if (s <= 0) return 0;
        L[i][j] = SQRT(s);
      } else {
        L[i][j] = s / L[j][j];
      }
    }
  for (int col = 0; col < 6; col++) {
    R y[6], x[6];
    for (int i = 0; i < 6; i++) {
      R s = (i == col) ? (R)1 : (R)0;
      for (int k = 0; k < i; k++) s -= L[i][k] * y[k];
      y[i] = s / L[i][i];
    }
    for (int i = 5; i >= 0; i--) {
      R s = y[i];
      for (int k = i + 1; k < 6; k++) s -= L[k][i] * x[k];
      x[i] = s / L[i][i];
    }
    for (int i = 0; i < 6; i++) Ainv[i * 6 + col] = x[i];
  }
  return 1;
}

/* kernels/solver_kernels.cu:358-399 — block-Jacobi inverse of (A_ii + 1e-4 I),
 * diagonal fallback when the Cholesky fails.  Returns the fallback count. */
static int F(precond)(int N, const int* row_ptr, const int* col_idx, const R* A, R* Minv) {
  int fallbacks = 0;
  for (int ni = 0; ni < N; ni++) {
    R D[36];
    memset(D, 0, sizeof(D));
    for (int r = row_ptr[ni]; r < row_ptr[ni + 1]; r++)
      if (col_idx[r] == ni) {
        for (int k = 0; k < 36; k++) D[k] = A[(size_t)r * 36 + k];
        break;
      }
    for (int k = 0; k < 6; k++) D[k * 6 + k] += (R)1e-4f;
    R* Mi = Minv + (size_t)ni * 36;
    if (!F(inv6_chol)(D, Mi)) {
      fallbacks++;
      for (int k = 0; k < 36; k++) Mi[k] = 0;
      for (int k = 0; k < 6; k++) Mi[k * 6 + k] = (R)1 / (D[k * 6 + k] + (R)1e-6f);
    }
  }
  return fallbacks;
}

/* kernels/solver_kernels.cu:406-432 */
static void F(spmv)(int N, const int* row_ptr, const int* col_idx, const R* A, const R* x, R* y,
                    int nthreads) {
#pragma omp parallel for num_threads(nthreads) schedule(static) if (nthreads > 1)
  for (int g = 0; g < N * 6; g++) {
    int ni = g / 6, row = g % 6;
    R s = 0;
    for (int bk = row_ptr[ni]; bk < row_ptr[ni + 1]; bk++) {
      const R* B = A + (size_t)bk * 36;
      const R* xj = x + (size_t)col_idx[bk] * 6;
      for (int c = 0; c < 6; c++) s += B[row * 6 + c] * xj[c];
    }
    y[g] = s;
  }
}

/* kernels/solver_kernels.cu:438-461 */
static void F(apply_precond)(int N, const R* Minv, const R* r, R* z) {
  for (int ni = 0; ni < N; ni++)
    for (int row = 0; row < 6; row++) {
      R acc = 0;
      for (int c = 0; c < 6; c++) acc += Minv[(size_t)ni * 36 + row * 6 + c] * r[ni * 6 + c];
      z[ni * 6 + row] = acc;
    }
}

static R F(dot)(const R* a, const R* b, int n, int nthreads) {
  R s = 0;
  if (nthreads > 1) {
#pragma omp parallel for num_threads(nthreads) reduction(+ : s) schedule(static)
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
  }
  for (int i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

/* kernels/solver_kernels.cu:616-687 — PCG from x = 0 with the reference's
 * guards: |p.Ap| < 1e-12 stops before the update, ||r|| < tol after it.
 * Returns the number of completed iterations; *final_r = ||r||. */
static int F(pcg)(int N, const int* row_ptr, const int* col_idx, const R* A, const R* bvec,
                  const R* Minv, int maxit, R tol, R* x, R* final_r, int nthreads) {
  int n = N * 6;
  R* r = (R*)malloc(sizeof(R) * n);
  R* z = (R*)malloc(sizeof(R) * n);
  R* p = (R*)malloc(sizeof(R) * n);
  R* Ap = (R*)malloc(sizeof(R) * n);
  for (int i = 0; i < n; i++) { x[i] = 0; r[i] = bvec[i]; }
  F(apply_precond)(N, Minv, r, z);
  for (int i = 0; i < n; i++) p[i] = z[i];
  R rz = F(dot)(r, z, n, nthreads);
  int used = 0;
  for (int it = 0; it < maxit; it++) {
    F(spmv)(N, row_ptr, col_idx, A, p, Ap, nthreads);
    R pAp = F(dot)(p, Ap, n, nthreads);
    if (FABS(pAp) < (R)1e-12f) { used = it; break; }
    R alpha = rz / pAp;
    for (int i = 0; i < n; i++) x[i] += alpha * p[i];
    for (int i = 0; i < n; i++) r[i] += -alpha * Ap[i];
    R rn = SQRT(F(dot)(r, r, n, nthreads));
    used = it + 1;
    if (rn < tol) break;
    F(apply_precond)(N, Minv, r, z);
    R rz_new = F(dot)(r, z, n, nthreads);
    R beta = rz_new / rz;
    for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    rz = rz_new;
  }
  *final_r = SQRT(F(dot)(r, r, n, nthreads));
  free(r); free(z); free(p); free(Ap);
  return used;
}

/* Assembles the full system (data term, ARAP, damping) at the given skinned
 * sources; returns the IRLS energy the assembly forms.  With nthreads > 1 the
 * data term is split over thread-private copies of A and b (the CPU baseline);
 * with nthreads == 1 the accumulation runs in correspondence order. */
static R F(assemble)(const cf_correspondence* corrs, const R* src3, int M, const cf_deform_node* nodes,
                     const cf_dual_quat* T, int N, const int* row_ptr, const int* col_idx,
                     R lambda_smooth, R lambda_damping, R* A, R* b, int nthreads) {
  int nnzb = row_ptr[N];
  memset(A, 0, sizeof(R) * (size_t)nnzb * 36);
  memset(b, 0, sizeof(R) * (size_t)N * 6);
  R e = 0;
  if (nthreads <= 1) {
    for (int c = 0; c < M; c++) {
      F(v3) s = src3 ? F(mk3)(src3[3 * c], src3[3 * c + 1], src3[3 * c + 2]) : F(ld3)(corrs[c].src);
      e += F(data_term)(&corrs[c], s, nodes, N, row_ptr, col_idx, A, b);
    }
  } else {
#pragma omp parallel num_threads(nthreads) reduction(+ : e)
    {
      R* Al = (R*)calloc((size_t)nnzb * 36, sizeof(R));
      R* bl = (R*)calloc((size_t)N * 6, sizeof(R));
#pragma omp for schedule(static)
      for (int c = 0; c < M; c++) {
        F(v3) s = src3 ? F(mk3)(src3[3 * c], src3[3 * c + 1], src3[3 * c + 2]) : F(ld3)(corrs[c].src);
        e += F(data_term)(&corrs[c], s, nodes, N, row_ptr, col_idx, Al, bl);
      }
#pragma omp critical
      {
        for (size_t i = 0; i < (size_t)nnzb * 36; i++) A[i] += Al[i];
        for (size_t i = 0; i < (size_t)N * 6; i++) b[i] += bl[i];
      }
      free(Al);
      free(bl);
    }
  }
  for (int ni = 0; ni < N; ni++) e += F(smooth_term)(ni, nodes, T, N, lambda_smooth, row_ptr, col_idx, A, b);
  F(damping)(N, row_ptr, col_idx, lambda_damping, A);
  return e;
}

/* Energy only (no system): the same terms the assembly forms. */
static R F(energy)(const cf_correspondence* corrs, const R* src3, int M, const cf_deform_node* nodes,
                   const cf_dual_quat* T, int N, R lambda_smooth, int nthreads) {
  R e = 0;
#pragma omp parallel for num_threads(nthreads) reduction(+ : e) schedule(static) if (nthreads > 1)
  for (int c = 0; c < M; c++) {
    const cf_correspondence* cc = &corrs[c];
    if (!cc->valid) continue;
    F(v3) s = F(mk3)(src3[3 * c], src3[3 * c + 1], src3[3 * c + 2]);
    F(v3) dst = F(ld3)(cc->dst), n = F(ld3)(cc->normal);
    R res = n.x * (s.x - dst.x) + n.y * (s.y - dst.y) + n.z * (s.z - dst.z);
    R fw = FMAX((R)cc->weight, (R)0) * F(huber)(res, (R)0.2f);
    if (fw <= (R)1e-8f) continue;
    e += fw * res * res;
  }
  /* ARAP energy: the residual and weight of smooth_term, without the system. */
  for (int ni = 0; ni < N; ni++) {
    const cf_deform_node* nd = &nodes[ni];
    for (int k = 0; k < nd->num_neighbors && k < CF_K_GRAPH; k++) {
      int nj = nd->neighbors[k];
      if (nj < 0 || nj >= N || nj <= ni) continue;
      R nw = FMAX((R)nd->neighbor_w[k], (R)0.05f);
      F(v3) xj = F(ld3)(nodes[nj].pos), xi = F(ld3)(nd->pos);
      F(dq) Ti = F(lddq)(&T[ni]), Tj = F(lddq)(&T[nj]);
      F(v3) Ti_xj = F(dq_transform_point_centered)(Ti, xj, xi);
      F(v3) Ti_xi = F(dq_transform_point_centered)(Ti, xi, xi);
      F(v3) Tj_xj = F(dq_transform_point_centered)(Tj, xj, xj);
      F(v3) rest = F(mk3)(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z);
      F(v3) curr = F(mk3)(Ti_xi.x - Tj_xj.x, Ti_xi.y - Tj_xj.y, Ti_xi.z - Tj_xj.z);
      R dr = SQRT(rest.x * rest.x + rest.y * rest.y + rest.z * rest.z);
      R dc = SQRT(curr.x * curr.x + curr.y * curr.y + curr.z * curr.z);
      R strain = FABS(dc - dr) / FMAX(dr, (R)1e-6f);
      R ratio = strain / (R)0.25f;
      R sw = EXP(-(ratio * ratio));
      F(v3) r = F(mk3)(Ti_xj.x - Tj_xj.x, Ti_xj.y - Tj_xj.y, Ti_xj.z - Tj_xj.z);
      R rn = SQRT(r.x * r.x + r.y * r.y + r.z * r.z);
      R el = lambda_smooth * nw * F(huber)(rn, (R)0.05f) * sw;
      if (el <= (R)1e-8f) continue;
      e += el * (r.x * r.x + r.y * r.y + r.z * r.z);
    }
  }
  return e;
}

static void F(skin_all)(const float* canon, const cf_correspondence* corrs, int M, const cf_deform_node* nodes,
                        const cf_dual_quat* T, int N, R* src3, int nthreads) {
#pragma omp parallel for num_threads(nthreads) schedule(static) if (nthreads > 1)
  for (int c = 0; c < M; c++) {
    F(v3) p = F(mk3)((R)canon[3 * c], (R)canon[3 * c + 1], (R)canon[3 * c + 2]);
    F(v3) s = F(warp_point)(p, nodes, T, N, corrs[c].node_ids, corrs[c].node_ws);
    src3[3 * c] = s.x; src3[3 * c + 1] = s.y; src3[3 * c + 2] = s.z;
  }
}

/* ======================= exported entry points ========================= */

CFO_EXPORT void F(cfo_exp_se3)(const float* tw, float* T16) {
  R t[6];
  for (int i = 0; i < 6; i++) t[i] = (R)tw[i];
  F(m4) T = F(exp_se3)(t);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) T16[i * 4 + j] = (float)T.m[i][j];
}

CFO_EXPORT void F(cfo_mat4_to_dq)(const float* T16, cf_dual_quat* out) {
  F(m4) T;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) T.m[i][j] = (R)T16[i * 4 + j];
  F(stdq)(out, F(mat4_to_dq)(&T));
}

CFO_EXPORT void F(cfo_dq_mul)(const cf_dual_quat* a, const cf_dual_quat* b, cf_dual_quat* out) {
  F(stdq)(out, F(dq_mul)(F(lddq)(a), F(lddq)(b)));
}

CFO_EXPORT void F(cfo_dq_centered)(const cf_dual_quat* a, const float* c, cf_dual_quat* out) {
  F(stdq)(out, F(dq_centered)(F(lddq)(a), F(mk3)(c[0], c[1], c[2])));
}

CFO_EXPORT void F(cfo_dq_transform_point)(const cf_dual_quat* a, const float* p, float* out) {
  F(v3) r = F(dq_transform_point)(F(lddq)(a), F(mk3)(p[0], p[1], p[2]));
  out[0] = (float)r.x; out[1] = (float)r.y; out[2] = (float)r.z;
}

CFO_EXPORT void F(cfo_dq_transform_point_centered)(const cf_dual_quat* a, const float* p, const float* c,
                                                  float* out) {
  F(v3) r = F(dq_transform_point_centered)(F(lddq)(a), F(mk3)(p[0], p[1], p[2]), F(mk3)(c[0], c[1], c[2]));
  out[0] = (float)r.x; out[1] = (float)r.y; out[2] = (float)r.z;
}

CFO_EXPORT void F(cfo_skin)(const float* canon, const int* ids, const float* ws, int M,
                            const cf_deform_node* nodes, const cf_dual_quat* T, int N, float* out) {
  for (int c = 0; c < M; c++) {
    F(v3) p = F(mk3)((R)canon[3 * c], (R)canon[3 * c + 1], (R)canon[3 * c + 2]);
    F(v3) s = F(warp_point)(p, nodes, T, N, ids + 4 * c, ws + 4 * c);
    out[3 * c] = (float)s.x; out[3 * c + 1] = (float)s.y; out[3 * c + 2] = (float)s.z;
  }
}

CFO_EXPORT void F(cfo_apply_twist)(cf_dual_quat* T, const float* dx, int N, float max_rot, float max_trans,
                                   float scale) {
  for (int i = 0; i < N; i++)
    F(stdq)(&T[i], F(twist_update)(F(lddq)(&T[i]), dx + 6 * i, (R)max_rot, (R)max_trans, (R)scale));
}

/* Assembly of one linearisation at corrs[].src; outputs in double. */
CFO_EXPORT double F(cfo_assemble)(const cf_correspondence* corrs, int M, const cf_deform_node* nodes,
                                  const cf_dual_quat* T, int N, const int* row_ptr, const int* col_idx,
                                  float lambda_smooth, float lambda_damping, double* A_out, double* b_out,
                                  int nthreads) {
  int nnzb = row_ptr[N];
  R* A = (R*)malloc(sizeof(R) * (size_t)nnzb * 36 + 1);
  R* b = (R*)malloc(sizeof(R) * (size_t)N * 6 + 1);
  R e = F(assemble)(corrs, NULL, M, nodes, T, N, row_ptr, col_idx, (R)lambda_smooth, (R)lambda_damping, A, b,
                    nthreads);
  for (size_t i = 0; i < (size_t)nnzb * 36; i++) A_out[i] = (double)A[i];
  for (size_t i = 0; i < (size_t)N * 6; i++) b_out[i] = (double)b[i];
  free(A);
  free(b);
  return (double)e;
}

/* One linearisation + PCG (GaussNewtonSolver::solve, solver_kernels.cu:543-570).
 * Returns the PCG iterations; dx in float.  stats_out[0] = energy,
 * stats_out[1] = final ||r||, stats_out[2] = preconditioner fallbacks. */
CFO_EXPORT int F(cfo_linearize_solve)(const cf_correspondence* corrs, int M, const cf_deform_node* nodes,
                                      const cf_dual_quat* T, int N, const int* row_ptr, const int* col_idx,
                                      const cf_gn_params* prm, float* dx, double* stats_out, int nthreads) {
  int nnzb = row_ptr[N];
  R* A = (R*)malloc(sizeof(R) * (size_t)nnzb * 36 + 1);
  R* b = (R*)malloc(sizeof(R) * (size_t)N * 6 + 1);
  R* Mi = (R*)malloc(sizeof(R) * (size_t)N * 36 + 1);
  R* x = (R*)malloc(sizeof(R) * (size_t)N * 6 + 1);
  R e = F(assemble)(corrs, NULL, M, nodes, T, N, row_ptr, col_idx, (R)prm->lambda_smooth,
                    (R)prm->lambda_damping, A, b, nthreads);
  int fb = F(precond)(N, row_ptr, col_idx, A, Mi);
  R fr = 0;
  int it = F(pcg)(N, row_ptr, col_idx, A, b, Mi, prm->pcg_iterations, (R)prm->pcg_tolerance, x, &fr, nthreads);
  for (int i = 0; i < N * 6; i++) dx[i] = (float)x[i];
  if (stats_out) {
    stats_out[0] = (double)e;
    stats_out[1] = (double)fr;
    stats_out[2] = (double)fb;
  }
  free(A); free(b); free(Mi); free(x);
  return it;
}

/* G Gauss-Newton iterations with re-skinning from canonical points and the
 * clamped DQ update after each PCG (the cf_gn_solve schedule).  T is updated
 * in place.  energies[G+1]: energy at each linearisation point and at the
 * end; pcg_iters[G]. */
CFO_EXPORT void F(cfo_gn_solve)(const float* canon, const cf_correspondence* corrs, int M,
                                const cf_deform_node* nodes, int N, const int* row_ptr, const int* col_idx,
                                const cf_gn_params* prm, float max_rot, float max_trans, float scale,
                                cf_dual_quat* T, double* energies, int* pcg_iters, int nthreads) {
  int nnzb = row_ptr[N];
  R* src3 = (R*)malloc(sizeof(R) * (size_t)M * 3 + 1);
  R* A = (R*)malloc(sizeof(R) * (size_t)nnzb * 36 + 1);
  R* b = (R*)malloc(sizeof(R) * (size_t)N * 6 + 1);
  R* Mi = (R*)malloc(sizeof(R) * (size_t)N * 36 + 1);
  R* x = (R*)malloc(sizeof(R) * (size_t)N * 6 + 1);
  float* dx = (float*)malloc(sizeof(float) * (size_t)N * 6 + 1);
  for (int g = 0; g < prm->gn_iterations; g++) {
    F(skin_all)(canon, corrs, M, nodes, T, N, src3, nthreads);
    R e = F(assemble)(corrs, src3, M, nodes, T, N, row_ptr, col_idx, (R)prm->lambda_smooth,
                      (R)prm->lambda_damping, A, b, nthreads);
    if (energies) energies[g] = (double)e;
    F(precond)(N, row_ptr, col_idx, A, Mi);
    R fr = 0;
    int it = F(pcg)(N, row_ptr, col_idx, A, b, Mi, prm->pcg_iterations, (R)prm->pcg_tolerance, x, &fr, nthreads);
    if (pcg_iters) pcg_iters[g] = it;
    for (int i = 0; i < N * 6; i++) dx[i] = (float)x[i];
    for (int i = 0; i < N; i++)
      F(stdq)(&T[i], F(twist_update)(F(lddq)(&T[i]), dx + 6 * i, (R)max_rot, (R)max_trans, (R)scale));
  }
  F(skin_all)(canon, corrs, M, nodes, T, N, src3, nthreads);
  if (energies)
    energies[prm->gn_iterations] = (double)F(energy)(corrs, src3, M, nodes, T, N, (R)prm->lambda_smooth, nthreads);
  free(src3); free(A); free(b); free(Mi); free(x); free(dx);
}

/* Energy at T from canonical points (re-skins first). */
CFO_EXPORT double F(cfo_energy)(const float* canon, const cf_correspondence* corrs, int M,
                                const cf_deform_node* nodes, const cf_dual_quat* T, int N, float lambda_smooth,
                                int nthreads) {
  R* src3 = (R*)malloc(sizeof(R) * (size_t)M * 3 + 1);
  F(skin_all)(canon, corrs, M, nodes, T, N, src3, nthreads);
  R e = F(energy)(corrs, src3, M, nodes, T, N, (R)lambda_smooth, nthreads);
  free(src3);
  return (double)e;
}
