/* Test infrastructure only: plain-C restatement of the reference's time step.
 * See mts_oracle.h.  Every expression keeps the operand order and grouping of
 * the reference statement it restates (cited per function), and the library is
 * built with -ffp-contract=off, so results are bit-identical to the reference
 * build on the same inputs.
 */
#include "mts_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Exact solutions.  Eq 0 restates src/equation/eq_0.cc (u = 80 inside, 100
 * outside, f = 0).  Eq 8 is the measured problem's solution
 *   inside  u = e^{-t} sin 2x cos 2y sin 2z,   outside u = e^{-t} (x^2+y^2+z^2)
 * with the evaluation order of the Eq8 class in oracle/ref_harness.cc. */
typedef struct {
  int eq;
  double bi, bo, E;
} eqn;

static eqn eq_at(const mts_oracle_problem* p, double t) {
  eqn e;
  e.eq = p->eq;
  e.bi = p->beta_in;
  e.bo = p->beta_out;
  e.E = exp(-t);
  return e;
}
static double inner_u(const eqn* e, double x, double y, double z) {
  if (e->eq == 0) return 80;
  return ((sin(2.0 * x) * cos(2.0 * y)) * sin(2.0 * z)) * e->E;
}
static double outer_u(const eqn* e, double x, double y, double z) {
  if (e->eq == 0) return 100;
  return ((x * x + y * y) + z * z) * e->E;
}
static double inner_f(const eqn* e, double x, double y, double z) {
  if (e->eq == 0) return 0.0;
  return (12.0 * e->bi - 1.0) * inner_u(e, x, y, z);
}
static double outer_f(const eqn* e, double x, double y, double z) {
  if (e->eq == 0) return 0.0;
  return -outer_u(e, x, y, z) - (6.0 * e->bo) * e->E;
}
/* [beta u_d] = beta_out * du_out/dd - beta_in * du_in/dd. */
static double jump_betau(const eqn* e, int d, double x, double y, double z) {
  if (e->eq == 0) {
    /* eq_0.cc:216-264: beta * 0 - beta * 0 */
    return e->bi * 0.0 - e->bo * 0.0;
  }
  double out_d, in_d;
  if (d == 0) {
    out_d = (2.0 * x) * e->E;
    in_d = (((2.0 * cos(2.0 * x)) * cos(2.0 * y)) * sin(2.0 * z)) * e->E;
  } else if (d == 1) {
    out_d = (2.0 * y) * e->E;
    in_d = (((-2.0 * sin(2.0 * x)) * sin(2.0 * y)) * sin(2.0 * z)) * e->E;
  } else {
    out_d = (2.0 * z) * e->E;
    in_d = (((2.0 * sin(2.0 * x)) * cos(2.0 * y)) * cos(2.0 * z)) * e->E;
  }
  return e->bo * out_d - e->bi * in_d;
}
/* Equation::Jump_u, src/equation/equation.cc:15-21 */
static double jump_u(const eqn* e, double x, double y, double z) {
  return outer_u(e, x, y, z) - inner_u(e, x, y, z);
}
/* Equation::Jump_betau_xi, src/equation/equation.cc:37-44 */
static double jump_betau_xi(const eqn* e, double x, double y, double z, double vx, double vy,
                            double vz) {
  return vx * jump_betau(e, 0, x, y, z) + vy * jump_betau(e, 1, x, y, z) +
         vz * jump_betau(e, 2, x, y, z);
}

/* ------------------------------------------------------------------------ */
/* 3x3 inverse by Crout LU with implicit pivoting, restating LU::LU, LU::solve
 * and LU::inverse (src/decomposition/lu.cc:15-71, 82-115, 146-161). */
static int lu_inverse3(const double a[9], double inv[9]) {
  const double TINY = 1.0e-40;
  double lu[3][3], vv[3], d = 1.0;
  int indx[3], n = 3, i, j, k, imax = 0;
  for (i = 0; i < n; i++)
    for (j = 0; j < n; j++) lu[i][j] = a[3 * i + j];
  for (i = 0; i < n; i++) {
    double big = 0.0, temp;
    for (j = 0; j < n; j++)
      if ((temp = fabs(lu[i][j])) > big) big = temp;
    if (big == 0.0) return 1;
    vv[i] = 1.0 / big;
  }
  for (k = 0; k < n; k++) {
    double big = 0.0, temp;
    for (i = k; i < n; i++) {
      temp = vv[i] * fabs(lu[i][k]);
      if (temp > big) {
        big = temp;
        imax = i;
      }
    }
    if (k != imax) {
      for (j = 0; j < n; j++) {
        temp = lu[imax][j];
        lu[imax][j] = lu[k][j];
        lu[k][j] = temp;
      }
      d = -d;
      vv[imax] = vv[k];
    }
    indx[k] = imax;
    if (lu[k][k] == 0.0) lu[k][k] = TINY;
    for (i = k + 1; i < n; i++) {
      temp = lu[i][k] /= lu[k][k];
      for (j = k + 1; j < n; j++) lu[i][j] -= temp * lu[k][j];
    }
  }
  (void)d;
  for (int col = 0; col < n; col++) {
    double x[3];
    for (i = 0; i < n; i++) x[i] = (i == col) ? 1.0 : 0.0;
    int ii = 0;
    for (i = 0; i < n; i++) {
      int ip = indx[i];
      double sum = x[ip];
      x[ip] = x[i];
      if (ii != 0) {
        for (j = ii - 1; j < i; j++) sum -= lu[i][j] * x[j];
      } else if (sum != 0.0) {
        ii = i + 1;
      }
      x[i] = sum;
    }
    for (i = n - 1; i >= 0; i--) {
      double sum = x[i];
      for (j = i + 1; j < n; j++) sum -= lu[i][j] * x[j];
      x[i] = sum / lu[i][i];
    }
    for (i = 0; i < n; i++) inv[3 * i + col] = x[i];
  }
  return 0;
}

/* ------------------------------------------------------------------------ */
typedef struct {
  const mts_oracle_problem* p;
  const int8_t* tags;
  const mts_oracle_crossing* cr;
  int nx, ny, nz;
  long nn;
  double h[3];
  double* xyz[3];
  int nline[3];     /* lines per direction (including boundary positions) */
  int* lstart[3];   /* CSR offsets over lines */
  int* lcross[3];   /* crossing indices, per line in left_loc order */
  double* jb;       /* per-crossing u_dir of the current step */
  double* gam;      /* TDMA workspace */
  double *a, *b, *c, *r, *ut;
} ctx;

static long node(const ctx* C, int ix, int iy, int iz) {
  return (long)ix + (long)C->nx * ((long)iy + (long)C->ny * iz);
}
static long dstride(const ctx* C, int d) {
  return d == 0 ? 1 : d == 1 ? C->nx : (long)C->nx * C->ny;
}
static int dlen(const ctx* C, int d) { return d == 0 ? C->nx : d == 1 ? C->ny : C->nz; }
/* Line (indx1, indx2) of direction d in the reference's index convention
 * (src/constant.h:83-89): x -> (iy, iz), y -> (ix, iz), z -> (ix, iy). */
static long line_base(const ctx* C, int d, int i1, int i2) {
  if (d == 0) return node(C, 0, i1, i2);
  if (d == 1) return node(C, i1, 0, i2);
  return node(C, i1, i2, 0);
}
static int line_id(const ctx* C, int d, int i1, int i2) {
  int n2 = d == 2 ? C->ny : C->nz;
  return i1 * n2 + i2;
}
static void node_xyz(const ctx* C, long m, double* x, double* y, double* z) {
  int ix = (int)(m % C->nx);
  long q = m / C->nx;
  int iy = (int)(q % C->ny);
  int iz = (int)(q / C->ny);
  *x = C->xyz[0][ix];
  *y = C->xyz[1][iy];
  *z = C->xyz[2][iz];
}

/* Operator_weights_{x,y,z} (src/temporal/douglas_adi.cc:1444-1539) for a
 * piecewise-constant beta: both half-point values come from the node's side. */
static void op_weights(const ctx* C, int d, long m, double vd[3]) {
  double beta = C->tags[m] > 0 ? C->p->beta_out : C->p->beta_in;
  double h = C->h[d];
  vd[0] = beta / (h * h);
  vd[1] = -(beta + beta) / (h * h);
  vd[2] = beta / (h * h);
}

static int build_lines(ctx* C, int ncr) {
  for (int d = 0; d < 3; d++) {
    int n1 = d == 0 ? C->ny : C->nx, n2 = d == 2 ? C->ny : C->nz;
    C->nline[d] = n1 * n2;
    C->lstart[d] = (int*)calloc((size_t)C->nline[d] + 1, sizeof(int));
    C->lcross[d] = (int*)malloc(sizeof(int) * (size_t)(ncr > 0 ? ncr : 1));
  }
  for (int k = 0; k < ncr; k++) {
    const mts_oracle_crossing* q = &C->cr[k];
    if (q->dir < 0 || q->dir > 2) return 2;
    int d = q->dir, n1 = d == 0 ? C->ny : C->nx, n2 = d == 2 ? C->ny : C->nz;
    if (q->indx1 < 1 || q->indx1 >= n1 - 1 || q->indx2 < 1 || q->indx2 >= n2 - 1) return 2;
    C->lstart[d][line_id(C, d, q->indx1, q->indx2) + 1]++;
  }
  for (int d = 0; d < 3; d++)
    for (int l = 0; l < C->nline[d]; l++) C->lstart[d][l + 1] += C->lstart[d][l];
  int* fill[3];
  for (int d = 0; d < 3; d++) {
    fill[d] = (int*)malloc(sizeof(int) * (size_t)C->nline[d]);
    memcpy(fill[d], C->lstart[d], sizeof(int) * (size_t)C->nline[d]);
  }
  for (int k = 0; k < ncr; k++) {
    const mts_oracle_crossing* q = &C->cr[k];
    int l = line_id(C, q->dir, q->indx1, q->indx2);
    C->lcross[q->dir][fill[q->dir][l]++] = k;
  }
  for (int d = 0; d < 3; d++) free(fill[d]);
  /* keep each line in increasing left_loc (the detection order of
   * Setup_Intersections, src/spatial/intersection.cc:79-291) */
  for (int d = 0; d < 3; d++)
    for (int l = 0; l < C->nline[d]; l++) {
      int s = C->lstart[d][l], e = C->lstart[d][l + 1];
      for (int i = s + 1; i < e; i++) {
        int v = C->lcross[d][i], j = i - 1;
        while (j >= s && C->cr[C->lcross[d][j]].left_loc > C->cr[v].left_loc) {
          C->lcross[d][j + 1] = C->lcross[d][j];
          j--;
        }
        C->lcross[d][j + 1] = v;
      }
      /* corner pairs must come in twos */
      for (int i = s; i < e;) {
        if (C->cr[C->lcross[d][i]].id > 0) {
          i += 1;
        } else {
          if (i + 1 >= e || C->cr[C->lcross[d][i + 1]].id >= 0) return 2;
          i += 2;
        }
      }
    }
  return 0;
}

static int ctx_init(ctx* C, const mts_oracle_problem* p, const int8_t* tags,
                    const mts_oracle_crossing* cr, int ncr) {
  memset(C, 0, sizeof *C);
  C->p = p;
  C->tags = tags;
  C->cr = cr;
  C->nx = p->nx;
  C->ny = p->ny;
  C->nz = p->nz;
  C->nn = (long)C->nx * C->ny * C->nz;
  /* Mesh::Mesh, src/mesh/mesh.cc:37-55 */
  C->h[0] = (p->xr - p->xl) / (C->nx - 1.0);
  C->h[1] = (p->yr - p->yl) / (C->ny - 1.0);
  C->h[2] = (p->zr - p->zl) / (C->nz - 1.0);
  double lo[3] = {p->xl, p->yl, p->zl};
  int n[3] = {C->nx, C->ny, C->nz};
  for (int d = 0; d < 3; d++) {
    C->xyz[d] = (double*)malloc(sizeof(double) * (size_t)n[d]);
    for (int i = 0; i < n[d]; i++) C->xyz[d][i] = lo[d] + i * C->h[d];
  }
  int nmax = C->nx > C->ny ? C->nx : C->ny;
  if (C->nz > nmax) nmax = C->nz;
  C->gam = (double*)malloc(sizeof(double) * (size_t)nmax);
  C->a = (double*)malloc(sizeof(double) * (size_t)nmax);
  C->b = (double*)malloc(sizeof(double) * (size_t)nmax);
  C->c = (double*)malloc(sizeof(double) * (size_t)nmax);
  C->r = (double*)malloc(sizeof(double) * (size_t)nmax);
  C->ut = (double*)malloc(sizeof(double) * (size_t)nmax);
  C->jb = (double*)calloc((size_t)(ncr > 0 ? ncr : 1), sizeof(double));
  /* line tables are built even without crossings (ncr == 0, cr NULL): the
     sweeps walk them for every line */
  return build_lines(C, ncr);
}

static void ctx_free(ctx* C) {
  for (int d = 0; d < 3; d++) {
    free(C->xyz[d]);
    free(C->lstart[d]);
    free(C->lcross[d]);
  }
  free(C->gam);
  free(C->a);
  free(C->b);
  free(C->c);
  free(C->r);
  free(C->ut);
  free(C->jb);
}

/* Intersections::Refresh_Jump (src/spatial/intersection.cc:2294-2490), the
 * part the time step reads: u_dir = (P^{-1})[d][0] * [beta u_xi]. */
static int refresh_jump(ctx* C, const eqn* e, int ncr) {
  for (int k = 0; k < ncr; k++) {
    const mts_oracle_crossing* q = &C->cr[k];
    double bxi = jump_betau_xi(e, q->coord[0], q->coord[1], q->coord[2], q->p[0], q->p[1], q->p[2]);
    double inv[9];
    if (lu_inverse3(q->p, inv)) return 2;
    C->jb[k] = inv[3 * q->dir + 0] * bxi;
  }
  return 0;
}

static double cjump_u(const ctx* C, const eqn* e, int k) {
  const mts_oracle_crossing* q = &C->cr[k];
  return jump_u(e, q->coord[0], q->coord[1], q->coord[2]);
}
/* Four-term corner jump combination, w[5..8] against ([u]_l, [bu]_l, [u]_r, [bu]_r). */
static double corner_jumps(const double* w, double jul, double jbl, double jur, double jbr) {
  return jul * w[5] + jbl * w[6] + jur * w[7] + jbr * w[8];
}

static void set_bc(const ctx* C, const eqn* e, double* uc) {
  /* Set_bc, src/temporal/lod.cc:216-236 (the ADI copies at
   * douglas_adi.cc:336-358 are the same loops). */
  int nx = C->nx, ny = C->ny, nz = C->nz;
  double* X = C->xyz[0];
  double* Y = C->xyz[1];
  double* Z = C->xyz[2];
  for (int ix = 0; ix < nx; ix++)
    for (int iy = 0; iy < ny; iy++) {
      uc[node(C, ix, iy, 0)] = outer_u(e, X[ix], Y[iy], Z[0]);
      uc[node(C, ix, iy, nz - 1)] = outer_u(e, X[ix], Y[iy], Z[nz - 1]);
    }
  for (int ix = 0; ix < nx; ix++)
    for (int iz = 0; iz < nz; iz++) {
      uc[node(C, ix, 0, iz)] = outer_u(e, X[ix], Y[0], Z[iz]);
      uc[node(C, ix, ny - 1, iz)] = outer_u(e, X[ix], Y[ny - 1], Z[iz]);
    }
  for (int iy = 0; iy < ny; iy++)
    for (int iz = 0; iz < nz; iz++) {
      uc[node(C, 0, iy, iz)] = outer_u(e, X[0], Y[iy], Z[iz]);
      uc[node(C, nx - 1, iy, iz)] = outer_u(e, X[nx - 1], Y[iy], Z[iz]);
    }
}

static int interior(const ctx* C, long m) {
  int ix = (int)(m % C->nx);
  long q = m / C->nx;
  int iy = (int)(q % C->ny);
  int iz = (int)(q / C->ny);
  return ix > 0 && ix < C->nx - 1 && iy > 0 && iy < C->ny - 1 && iz > 0 && iz < C->nz - 1;
}

/* Explicit 3-point operator along d with MIB rows, written to out at every
 * interior node.
 *   mode 0 (Douglas-ADI RHS, douglas_adi.cc:93-210 / 516-640 / 809-930):
 *          out = k * sum, k = +dt or -dt; the jumps live in the source term.
 *   mode 1 (LOD-CN / TS, lod.cc:309-505 and trapezoidal.cc D_xx_r):
 *          out = (coef*dt) * sum with the jump terms inside sum, then
 *          out += in at interior nodes.                                      */
static void explicit_op(ctx* C, int d, int mode, double k, const eqn* e, const double* in,
                        double* out) {
  long s = dstride(C, d);
  for (long m = 0; m < C->nn; m++) {
    if (!interior(C, m)) continue;
    double vd[3], sum = 0;
    op_weights(C, d, m, vd);
    for (int i = -1; i < 2; i++) sum += in[m + i * s] * vd[i + 1];
    out[m] = k * sum;
  }
  int n1 = d == 0 ? C->ny : C->nx, n2 = d == 2 ? C->ny : C->nz;
  for (int i1 = 1; i1 < n1 - 1; i1++)
    for (int i2 = 1; i2 < n2 - 1; i2++) {
      int l = line_id(C, d, i1, i2);
      long base = line_base(C, d, i1, i2);
      int ip = C->lstart[d][l], end = C->lstart[d][l + 1];
      while (ip < end) {
        int k0 = C->lcross[d][ip];
        const mts_oracle_crossing* q = &C->cr[k0];
        double vd[3], sum;
        if (q->id > 0) {
          double ju = mode ? cjump_u(C, e, k0) : 0, jb = mode ? C->jb[k0] : 0;
          int L = q->left_loc;
          long m = base + (long)L * s;
          op_weights(C, d, m, vd);
          sum = 0;
          for (int i = -1; i < 1; i++) sum += vd[i + 1] * in[m + i * s];
          for (int i = 0; i < 4; i++) sum += vd[2] * in[base + (long)(L - 1 + i) * s] * q->weir[i];
          if (mode) sum += vd[2] * (ju * q->weir[4] + jb * q->weir[5]);
          out[m] = mode ? k * sum : sum * k;
          m += s;
          op_weights(C, d, m, vd);
          sum = 0;
          for (int i = 0; i < 2; i++) sum += vd[i + 1] * in[m + i * s];
          for (int i = 0; i < 4; i++) sum += vd[0] * in[base + (long)(L - 1 + i) * s] * q->weil[i];
          if (mode) sum += vd[0] * (ju * q->weil[4] + jb * q->weil[5]);
          out[m] = mode ? k * sum : sum * k;
          ip += 1;
        } else {
          int k1 = C->lcross[d][ip + 1];
          const mts_oracle_crossing* qr = &C->cr[k1];
          double jul = 0, jur = 0, jbl = 0, jbr = 0;
          if (mode) {
            jul = cjump_u(C, e, k0);
            jur = cjump_u(C, e, k1);
            jbl = C->jb[k0];
            jbr = C->jb[k1];
          }
          int L = q->left_loc, R = qr->left_loc;
          long m = base + (long)L * s;
          op_weights(C, d, m, vd);
          sum = 0;
          for (int i = -1; i < 1; i++) sum += vd[i + 1] * in[m + i * s];
          for (int i = 0; i < 5; i++) sum += vd[2] * in[base + (long)(L - 1 + i) * s] * q->weir[i];
          if (mode) sum += vd[2] * corner_jumps(q->weir, jul, jbl, jur, jbr);
          out[m] = mode ? k * sum : sum * k;
          m += s;
          op_weights(C, d, m, vd);
          sum = 0;
          for (int i = 0; i < 5; i++) sum += vd[0] * in[base + (long)(L - 1 + i) * s] * q->weil[i];
          if (mode) {
            sum += vd[0] * corner_jumps(q->weil, jul, jbl, jur, jbr);
            sum += vd[1] * in[m];
            for (int i = 0; i < 5; i++) sum += vd[2] * in[base + (long)(R - 2 + i) * s] * qr->weir[i];
            sum += vd[2] * corner_jumps(qr->weir, jul, jbl, jur, jbr);
          } else {
            sum += vd[1] * in[m];
            for (int i = 0; i < 5; i++) sum += vd[2] * in[base + (long)(R - 2 + i) * s] * qr->weir[i];
          }
          out[m] = mode ? k * sum : sum * k;
          m += s;
          op_weights(C, d, m, vd);
          sum = 0;
          for (int i = 0; i < 2; i++) sum += vd[i + 1] * in[m + i * s];
          for (int i = 0; i < 5; i++) sum += vd[0] * in[base + (long)(R - 2 + i) * s] * qr->weil[i];
          if (mode) sum += vd[0] * corner_jumps(qr->weil, jul, jbl, jur, jbr);
          out[m] = mode ? k * sum : sum * k;
          ip += 2;
        }
      }
    }
  if (mode)
    for (long m = 0; m < C->nn; m++)
      if (interior(C, m)) out[m] += in[m];
}

/* Convert2Tri_irr (douglas_adi.cc:1554-1577): eliminate the two extra
 * columns of a 2x5 MIB row block. */
static void convert_irr(int L, double row[2][5], double* a, double* b, double* c, double* r) {
  double rate = row[1][0] / row[0][0];
  for (int i = 0; i < 5; i++) row[1][i] -= rate * row[0][i];
  rate = row[0][3] / row[1][3];
  for (int i = 0; i < 5; i++) row[0][i] -= rate * row[1][i];
  for (int i = 0; i < 2; i++) {
    a[L + i] = row[i][i];
    b[L + i] = row[i][i + 1];
    c[L + i] = row[i][i + 2];
    r[L + i] = row[i][4];
  }
}

/* Convert2Tri_cor (douglas_adi.cc:1637-1675): 3x6 corner block. */
static void convert_cor(int L, double row[3][6], double* a, double* b, double* c, double* r) {
  double rate[3];
  rate[1] = row[1][0] / row[0][0];
  rate[2] = row[2][0] / row[0][0];
  for (int i = 0; i < 6; i++) {
    row[1][i] -= rate[1] * row[0][i];
    row[2][i] -= rate[2] * row[0][i];
  }
  rate[0] = row[0][4] / row[2][4];
  rate[1] = row[1][4] / row[2][4];
  for (int i = 0; i < 6; i++) {
    row[0][i] -= rate[0] * row[2][i];
    row[1][i] -= rate[1] * row[2][i];
  }
  rate[2] = row[2][1] / row[1][1];
  for (int i = 0; i < 6; i++) row[2][i] -= rate[2] * row[1][i];
  rate[0] = row[0][3] / row[1][3];
  for (int i = 0; i < 6; i++) row[0][i] -= rate[0] * row[1][i];
  for (int i = 0; i < 3; i++) {
    a[L + i] = row[i][i];
    b[L + i] = row[i][i + 1];
    c[L + i] = row[i][i + 2];
    r[L + i] = row[i][5];
  }
}

/* TDMA (douglas_adi.cc:1784-1807), Numerical-Recipes tridag. */
static int tdma(int n, const double* a, const double* b, const double* c, const double* r,
                double* u, double* gam) {
  double bet;
  if (b[0] == 0.0) return 1;
  u[0] = r[0] / (bet = b[0]);
  for (int j = 1; j < n; j++) {
    gam[j] = c[j - 1] / bet;
    bet = b[j] - a[j] * gam[j];
    if (bet == 0.0) return 1;
    u[j] = (r[j] - a[j] * u[j - 1]) / bet;
  }
  for (int j = n - 2; j >= 0; j--) u[j] -= gam[j + 1] * u[j + 1];
  return 0;
}

/* Implicit sweep (I - cdt * beta D_dd) along every interior line of d, in
 * place on uc.  cdt = dt (Douglas-ADI, LOD-IE) or 0.5*dt (LOD-CN, TS).
 * jumps = 0: right-hand sides of MIB rows are the array values (Douglas-ADI,
 * douglas_adi.cc:361-514); jumps = 1: the jump terms are added to them
 * (D_xx_l, lod.cc:887-1100). */
static int implicit_sweep(ctx* C, int d, double cdt, int jumps, const eqn* e, double* uc) {
  long s = dstride(C, d);
  int n = dlen(C, d);
  int n1 = d == 0 ? C->ny : C->nx, n2 = d == 2 ? C->ny : C->nz;
  double *a = C->a, *b = C->b, *c = C->c, *r = C->r, *ut = C->ut;
  for (int i1 = 1; i1 < n1 - 1; i1++)
    for (int i2 = 1; i2 < n2 - 1; i2++) {
      long base = line_base(C, d, i1, i2);
      double vd[3];
      a[0] = 0.0;
      b[0] = 1.0;
      c[0] = 0.0;
      for (int j = 1; j < n - 1; j++) {
        op_weights(C, d, base + j * s, vd);
        a[j] = -cdt * vd[0];
        b[j] = 1 - cdt * vd[1];
        c[j] = -cdt * vd[2];
      }
      a[n - 1] = 0.0;
      b[n - 1] = 1.0;
      c[n - 1] = 0.0;
      for (int j = 0; j < n; j++) r[j] = uc[base + j * s];

      int l = line_id(C, d, i1, i2);
      int ip = C->lstart[d][l], end = C->lstart[d][l + 1];
      while (ip < end) {
        int k0 = C->lcross[d][ip];
        const mts_oracle_crossing* q = &C->cr[k0];
        if (q->id > 0) {
          double row[2][5];
          memset(row, 0, sizeof row);
          double ju = jumps ? cjump_u(C, e, k0) : 0, jb = jumps ? C->jb[k0] : 0;
          int j = q->left_loc;
          op_weights(C, d, base + j * s, vd);
          row[0][0] = -cdt * vd[0];
          row[0][1] = 1 - cdt * vd[1];
          for (int i = 0; i < 4; i++) row[0][i] += -cdt * vd[2] * q->weir[i];
          row[0][4] = jumps ? uc[base + j * s] + cdt * vd[2] * (ju * q->weir[4] + jb * q->weir[5])
                            : uc[base + j * s];
          j += 1;
          op_weights(C, d, base + j * s, vd);
          row[1][2] = 1 - cdt * vd[1];
          row[1][3] = -cdt * vd[2];
          for (int i = 0; i < 4; i++) row[1][i] += -cdt * vd[0] * q->weil[i];
          row[1][4] = jumps ? uc[base + j * s] + cdt * vd[0] * (ju * q->weil[4] + jb * q->weil[5])
                            : uc[base + j * s];
          convert_irr(q->left_loc, row, a, b, c, r);
          ip += 1;
        } else {
          int k1 = C->lcross[d][ip + 1];
          const mts_oracle_crossing* qr = &C->cr[k1];
          double row[3][6];
          memset(row, 0, sizeof row);
          double jul = 0, jur = 0, jbl = 0, jbr = 0;
          if (jumps) {
            jul = cjump_u(C, e, k0);
            jur = cjump_u(C, e, k1);
            jbl = C->jb[k0];
            jbr = C->jb[k1];
          }
          int j = q->left_loc;
          op_weights(C, d, base + j * s, vd);
          row[0][0] = -cdt * vd[0];
          row[0][1] = 1 - cdt * vd[1];
          for (int i = 0; i < 5; i++) row[0][i] -= cdt * vd[2] * q->weir[i];
          row[0][5] = jumps ? uc[base + j * s] + cdt * vd[2] * corner_jumps(q->weir, jul, jbl, jur, jbr)
                            : uc[base + j * s];
          j += 1;
          op_weights(C, d, base + j * s, vd);
          row[1][2] = 1 - cdt * vd[1];
          for (int i = 0; i < 5; i++) row[1][i] -= cdt * vd[0] * q->weil[i];
          row[1][5] = jumps ? uc[base + j * s] + cdt * vd[0] * corner_jumps(q->weil, jul, jbl, jur, jbr)
                            : uc[base + j * s];
          for (int i = 0; i < 5; i++) row[1][i] -= cdt * vd[2] * qr->weir[i];
          if (jumps) row[1][5] += cdt * vd[2] * corner_jumps(qr->weir, jul, jbl, jur, jbr);
          j += 1;
          op_weights(C, d, base + j * s, vd);
          row[2][3] = 1 - cdt * vd[1];
          row[2][4] = -cdt * vd[2];
          for (int i = 0; i < 5; i++) row[2][i] -= cdt * vd[0] * qr->weil[i];
          row[2][5] = jumps ? uc[base + j * s] + cdt * vd[0] * corner_jumps(qr->weil, jul, jbl, jur, jbr)
                            : uc[base + j * s];
          convert_cor(q->left_loc, row, a, b, c, r);
          ip += 2;
        }
      }
      if (tdma(n, a, b, c, r, ut, C->gam)) return 1;
      for (int j = 0; j < n; j++) uc[base + j * s] = ut[j];
    }
  return 0;
}

/* Douglas_ADI::Src_2nd (douglas_adi.cc:1123-1428): f by node tag, then the
 * MIB jump terms of the x, y and z crossings in that order. */
static void adi_source(ctx* C, const eqn* e, double* src) {
  for (long m = 0; m < C->nn; m++) {
    double x, y, z;
    node_xyz(C, m, &x, &y, &z);
    src[m] = C->tags[m] == 1 ? outer_f(e, x, y, z) : inner_f(e, x, y, z);
  }
  for (int d = 0; d < 3; d++) {
    long s = dstride(C, d);
    int n1 = d == 0 ? C->ny : C->nx, n2 = d == 2 ? C->ny : C->nz;
    for (int i1 = 1; i1 < n1 - 1; i1++)
      for (int i2 = 1; i2 < n2 - 1; i2++) {
        int l = line_id(C, d, i1, i2);
        long base = line_base(C, d, i1, i2);
        int ip = C->lstart[d][l], end = C->lstart[d][l + 1];
        while (ip < end) {
          int k0 = C->lcross[d][ip];
          const mts_oracle_crossing* q = &C->cr[k0];
          double vd[3];
          if (q->id > 0) {
            double ju = cjump_u(C, e, k0), jb = C->jb[k0];
            long m = base + (long)q->left_loc * s;
            op_weights(C, d, m, vd);
            src[m] += vd[2] * (ju * q->weir[4] + jb * q->weir[5]);
            m += s;
            op_weights(C, d, m, vd);
            src[m] += vd[0] * (ju * q->weil[4] + jb * q->weil[5]);
            ip += 1;
          } else {
            int k1 = C->lcross[d][ip + 1];
            const mts_oracle_crossing* qr = &C->cr[k1];
            double jul = cjump_u(C, e, k0), jur = cjump_u(C, e, k1);
            double jbl = C->jb[k0], jbr = C->jb[k1];
            long m = base + (long)q->left_loc * s;
            op_weights(C, d, m, vd);
            src[m] += vd[2] * corner_jumps(q->weir, jul, jbl, jur, jbr);
            m += s;
            op_weights(C, d, m, vd);
            src[m] += vd[0] * corner_jumps(q->weil, jul, jbl, jur, jbr);
            src[m] += vd[2] * corner_jumps(qr->weir, jul, jbl, jur, jbr);
            m += s;
            op_weights(C, d, m, vd);
            src[m] += vd[0] * corner_jumps(qr->weil, jul, jbl, jur, jbr);
            ip += 2;
          }
        }
      }
  }
}

/* LOD::Src_2nd / TS::Src_2nd (lod.cc:1509-1531): f by node tag only. */
static void plain_source(ctx* C, const eqn* e, double* src) {
  for (long m = 0; m < C->nn; m++) {
    double x, y, z;
    node_xyz(C, m, &x, &y, &z);
    src[m] = C->tags[m] == 1 ? outer_f(e, x, y, z) : inner_f(e, x, y, z);
  }
}

/* Douglas_ADI::Solve_2nd, douglas_adi.cc:66-1110. */
static int adi_step(ctx* C, double t1, int ncr, double* uh, double* w[4]) {
  eqn e = eq_at(C->p, t1);
  double dt = C->p->dt;
  double *uhs = w[0], *uhs2 = w[1], *src = w[2], *tmp = w[3];
  if (refresh_jump(C, &e, ncr)) return 2;
  adi_source(C, &e, src);
  explicit_op(C, 1, 0, dt, &e, uh, uhs);
  explicit_op(C, 2, 0, dt, &e, uh, uhs2);
  for (long m = 0; m < C->nn; m++)
    if (interior(C, m)) uhs[m] += uhs2[m];
  for (long m = 0; m < C->nn; m++)
    if (interior(C, m)) uhs[m] += uh[m];
  for (long m = 0; m < C->nn; m++)
    if (interior(C, m)) uhs[m] += dt * src[m];
  set_bc(C, &e, uhs);
  if (implicit_sweep(C, 0, dt, 0, &e, uhs)) return 1;
  /* second stage: uhss = -dt*D_yy u^n + u* */
  explicit_op(C, 1, 0, -dt, &e, uh, tmp);
  for (long m = 0; m < C->nn; m++)
    if (interior(C, m)) tmp[m] += uhs[m];
  set_bc(C, &e, tmp);
  if (implicit_sweep(C, 1, dt, 0, &e, tmp)) return 1;
  /* third stage: uh1 = -dt*D_zz u^n + u** */
  explicit_op(C, 2, 0, -dt, &e, uh, uhs2);
  for (long m = 0; m < C->nn; m++)
    if (interior(C, m)) uhs2[m] += tmp[m];
  set_bc(C, &e, uhs2);
  if (implicit_sweep(C, 2, dt, 0, &e, uhs2)) return 1;
  memcpy(uh, uhs2, sizeof(double) * (size_t)C->nn);
  return 0;
}

/* LOD::Solve_2nd, lod.cc:44-205; cn = 0 implicit Euler, 1 Crank-Nicolson. */
static int lod_step(ctx* C, double t1, int ncr, int cn, double* uh, double* w[4]) {
  eqn e = eq_at(C->p, t1);
  double dt = C->p->dt;
  double coef = cn ? 0.5 : 1;
  double cdt = coef * dt;
  double *v = w[0], *v2 = w[1], *src = w[2];
  if (refresh_jump(C, &e, ncr)) return 2;
  plain_source(C, &e, src);
  double* cur = uh;
  double* nxt = v;
  for (int d = 0; d < 3; d++) {
    if (cn) {
      explicit_op(C, d, 1, 0.5 * dt, &e, cur, nxt);
    } else {
      memcpy(nxt, cur, sizeof(double) * (size_t)C->nn);
    }
    set_bc(C, &e, nxt);
    if (implicit_sweep(C, d, cdt, 1, &e, nxt)) return 1;
    cur = nxt;
    nxt = (nxt == v) ? v2 : v;
  }
  for (long m = 0; m < C->nn; m++) uh[m] = cur[m] + dt * src[m];
  return 0;
}

/* TS::Solve_2nd, trapezoidal.cc:46-272. */
static int ts_step(ctx* C, double t1, int ncr, double* uh, double* w[4]) {
  double dt = C->p->dt;
  eqn e0 = eq_at(C->p, t1 - dt);
  eqn eh = eq_at(C->p, t1 - 0.5 * dt);
  eqn e1 = eq_at(C->p, t1);
  double *v = w[0], *v2 = w[1], *src = w[2];
  if (refresh_jump(C, &e1, ncr)) return 2;
  explicit_op(C, 0, 1, 0.5 * dt, &e1, uh, v);
  set_bc(C, &eh, v);
  explicit_op(C, 1, 1, 0.5 * dt, &e1, v, v2);
  set_bc(C, &eh, v2);
  explicit_op(C, 2, 1, 0.5 * dt, &e1, v2, v);
  set_bc(C, &eh, v);
  plain_source(C, &e0, src);
  for (long m = 0; m < C->nn; m++) v[m] = v[m] + 0.5 * dt * src[m];
  plain_source(C, &e1, src);
  for (long m = 0; m < C->nn; m++) v[m] = v[m] + 0.5 * dt * src[m];
  set_bc(C, &e1, v);
  if (implicit_sweep(C, 2, 0.5 * dt, 1, &e1, v)) return 1;
  set_bc(C, &e1, v);
  if (implicit_sweep(C, 1, 0.5 * dt, 1, &e1, v)) return 1;
  set_bc(C, &e1, v);
  if (implicit_sweep(C, 0, 0.5 * dt, 1, &e1, v)) return 1;
  memcpy(uh, v, sizeof(double) * (size_t)C->nn);
  return 0;
}

int mts_oracle_init(const mts_oracle_problem* p, const int8_t* tags, double t, double* u) {
  ctx C;
  ctx_init(&C, p, tags, NULL, 0);
  eqn e = eq_at(p, t);
  for (long m = 0; m < C.nn; m++) {
    double x, y, z;
    node_xyz(&C, m, &x, &y, &z);
    u[m] = tags[m] == 1 ? outer_u(&e, x, y, z) : inner_u(&e, x, y, z);
  }
  ctx_free(&C);
  return 0;
}

int mts_oracle_run(const mts_oracle_problem* p, const int8_t* tags, const mts_oracle_crossing* cr,
                   int32_t ncr, int32_t method, double t0, int32_t steps, double* u) {
  ctx C;
  int rc = ctx_init(&C, p, tags, cr, ncr);
  if (rc) {
    ctx_free(&C);
    return rc;
  }
  double* w[4];
  for (int i = 0; i < 4; i++) w[i] = (double*)calloc((size_t)C.nn, sizeof(double));
  double t = t0;
  for (int s = 0; s < steps && rc == 0; s++) {
    t += p->dt;
    if (method == MTS_ORACLE_ADI)
      rc = adi_step(&C, t, ncr, u, w);
    else if (method == MTS_ORACLE_LOD_IE)
      rc = lod_step(&C, t, ncr, 0, u, w);
    else if (method == MTS_ORACLE_LOD_CN)
      rc = lod_step(&C, t, ncr, 1, u, w);
    else if (method == MTS_ORACLE_TS)
      rc = ts_step(&C, t, ncr, u, w);
    else
      rc = 2;
  }
  for (int i = 0; i < 4; i++) free(w[i]);
  ctx_free(&C);
  return rc;
}

int mts_oracle_norms(const mts_oracle_problem* p, const int8_t* tags, double t, const double* u,
                     double* lmax, double* l2, int32_t* am) {
  ctx C;
  ctx_init(&C, p, tags, NULL, 0);
  eqn e = eq_at(p, t);
  double mx = 0, s2 = 0;
  am[0] = am[1] = am[2] = 0;
  for (int ix = 0; ix < C.nx; ix++)
    for (int iy = 0; iy < C.ny; iy++)
      for (int iz = 0; iz < C.nz; iz++) {
        long m = node(&C, ix, iy, iz);
        double X = C.xyz[0][ix], Y = C.xyz[1][iy], Z = C.xyz[2][iz];
        double temp = fabs(u[m] - (tags[m] == 1 ? outer_u(&e, X, Y, Z) : inner_u(&e, X, Y, Z)));
        if (temp > mx) {
          mx = temp;
          am[0] = ix;
          am[1] = iy;
          am[2] = iz;
        }
        s2 += temp * temp;
      }
  *lmax = mx;
  *l2 = sqrt(s2 / (1.0 * C.nx * C.ny * C.nz));
  ctx_free(&C);
  return 0;
}
