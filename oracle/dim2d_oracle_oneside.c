/*
 * dim2d_oracle_oneside.c -- the one-sided Mattsson operator sets used near
 * boundaries (wall corners, open-boundary transverse fluxes).  Each set
 * extends the interior set and overrides a few operators, exactly as the
 * reference's type extensions do.  TEST INFRASTRUCTURE ONLY.
 *
 * src/sd_operators/mattsson_operators/sd_operators_{x,y}_oneside_{L0,L1,R1,R0}_class.f
 */
#include "dim2d_oracle_internal.h"

/* ---------------- x_oneside_L0 (sd_operators_x_oneside_L0_class.f) ---- */
/* :162-182 */
static double f_xL0(const ov *n, int i, int j, primary_proc p) {
  return 1.5 * p(n, i, j) - 0.5 * p(n, i + 1, j);
}
/* :215-240 */
static double dfdx_xL0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / dx * (-2.0 * p(n, i, j) + 3.0 * p(n, i + 1, j) - p(n, i + 2, j));
}
/* :276-302 */
static double dfdx_nl_xL0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dx *
         (-2.0 * p(n, i, j, dx, dy, gradient_x_x_oneside_L0, gradient_y_interior) +
          3.0 * p(n, i + 1, j, dx, dy, gradient_x_interior, gradient_y_interior) -
          p(n, i + 2, j, dx, dy, gradient_x_interior, gradient_y_interior));
}
/* :335-363 */
static double dfdy_xL0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / (2.0 * dy) *
         (-1.5 * p(n, i, j - 1) + 0.5 * p(n, i + 1, j - 1) + 1.5 * p(n, i, j + 1) -
          0.5 * p(n, i + 1, j + 1));
}
/* :396-428 */
static double d2fdx2_xL0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 0.5 / (dx * dx) *
         (+3.0 * p(n, i, j) - 5.0 * p(n, i + 1, j) - p(n, i + 2, j) + 5.0 * p(n, i + 3, j) -
          2.0 * p(n, i + 4, j));
}
/* :462-503 */
static double d2fdy2_xL0(const ov *n, int i, int j, primary_proc p, double dy) {
  return (1.0 / (dy * dy)) *
         (1.5 * p(n, i, j - 1) - 0.5 * p(n, i + 1, j - 1) -
          2.0 * (1.5 * p(n, i, j) - 0.5 * p(n, i + 1, j)) + 1.5 * p(n, i, j + 1) -
          0.5 * p(n, i + 1, j + 1));
}
/* :540-574 */
static double d2fdxdy_xL0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (2.0 * p(n, i, j - 1) - 3.0 * p(n, i + 1, j - 1) + p(n, i + 2, j - 1) -
          2.0 * p(n, i, j + 1) + 3.0 * p(n, i + 1, j + 1) - p(n, i + 2, j + 1)) *
         0.5 / (dy * dx);
}
/* :607-636 */
static double dgdx_xL0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / dx *
         (-0.5 * p(n, i, j - 1) - 0.5 * p(n, i, j) + 0.5 * p(n, i + 1, j - 1) +
          0.5 * p(n, i + 1, j));
}
/* :671-699 */
static double dgdy_nl_xL0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dy * (-p(n, i, j - 1, dx, dy, gradient_x_x_oneside_L0, gradient_y_interior) +
                     p(n, i, j, dx, dy, gradient_x_x_oneside_L0, gradient_y_interior));
}
/* :733-772 */
static double d2gdx2_xL0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / (dx * dx) *
         (0.5 * p(n, i, j - 1) + 0.5 * p(n, i, j) -
          2.0 * (+0.5 * p(n, i + 1, j - 1) + 0.5 * p(n, i + 1, j)) + 0.5 * p(n, i + 2, j - 1) +
          0.5 * p(n, i + 2, j));
}
/* :809-841 */
static double d2gdxdy_xL0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (p(n, i, j - 1) - p(n, i, j) - p(n, i + 1, j - 1) + p(n, i + 1, j)) * 1.0 / (dx * dy);
}

/* ---------------- x_oneside_L1 (sd_operators_x_oneside_L1_class.f) ---- */
/* :160-184 */
static double dfdx_nl_xL1(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dx * (-p(n, i - 1, j, dx, dy, gradient_x_x_oneside_L0, gradient_y_interior) +
                     p(n, i, j, dx, dy, gradient_x_interior, gradient_y_interior));
}
/* :217-249 */
static double d2fdx2_xL1(const ov *n, int i, int j, primary_proc p, double dx) {
  return 0.5 / (dx * dx) *
         (+p(n, i - 1, j) + p(n, i, j) - 7.0 * p(n, i + 1, j) + 7.0 * p(n, i + 2, j) -
          2.0 * p(n, i + 3, j));
}

/* ---------------- x_oneside_R1 (sd_operators_x_oneside_R1_class.f) ---- */
/* :157-181 */
static double dfdx_nl_xR1(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dx * (-p(n, i - 1, j, dx, dy, gradient_x_interior, gradient_y_interior) +
                     p(n, i, j, dx, dy, gradient_x_x_oneside_R0, gradient_y_interior));
}
/* :214-246 */
static double d2fdx2_xR1(const ov *n, int i, int j, primary_proc p, double dx) {
  return 0.5 / (dx * dx) *
         (-2.0 * p(n, i - 4, j) + 7.0 * p(n, i - 3, j) - 7.0 * p(n, i - 2, j) + p(n, i - 1, j) +
          p(n, i, j));
}

/* ---------------- x_oneside_R0 (sd_operators_x_oneside_R0_class.f) ---- */
/* :162-182 */
static double f_xR0(const ov *n, int i, int j, primary_proc p) {
  return -0.5 * p(n, i - 2, j) + 1.5 * p(n, i - 1, j);
}
/* :215-240 */
static double dfdx_xR0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / dx * (p(n, i - 3, j) - 3.0 * p(n, i - 2, j) + 2.0 * p(n, i - 1, j));
}
/* :276-302 */
static double dfdx_nl_xR0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dx *
         (p(n, i - 3, j, dx, dy, gradient_x_interior, gradient_y_interior) -
          3.0 * p(n, i - 2, j, dx, dy, gradient_x_interior, gradient_y_interior) +
          2.0 * p(n, i - 1, j, dx, dy, gradient_x_x_oneside_R0, gradient_y_interior));
}
/* :335-363 */
static double dfdy_xR0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / (2.0 * dy) *
         (+0.5 * p(n, i - 2, j - 1) - 1.5 * p(n, i - 1, j - 1) - 0.5 * p(n, i - 2, j + 1) +
          1.5 * p(n, i - 1, j + 1));
}
/* :396-428 */
static double d2fdx2_xR0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 0.5 / (dx * dx) *
         (-2.0 * p(n, i - 5, j) + 5.0 * p(n, i - 4, j) - p(n, i - 3, j) - 5.0 * p(n, i - 2, j) +
          3.0 * p(n, i - 1, j));
}
/* :462-503 */
static double d2fdy2_xR0(const ov *n, int i, int j, primary_proc p, double dy) {
  return (1.0 / (dy * dy)) *
         (-0.5 * p(n, i - 2, j - 1) + 1.5 * p(n, i - 1, j - 1) -
          2.0 * (-0.5 * p(n, i - 2, j) + 1.5 * p(n, i - 1, j)) - 0.5 * p(n, i - 2, j + 1) +
          1.5 * p(n, i - 1, j + 1));
}
/* :540-574 */
static double d2fdxdy_xR0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (-p(n, i - 3, j - 1) + 3.0 * p(n, i - 2, j - 1) - 2.0 * p(n, i - 1, j - 1) +
          p(n, i - 3, j + 1) - 3.0 * p(n, i - 2, j + 1) + 2.0 * p(n, i - 1, j + 1)) *
         0.5 / (dy * dx);
}
/* :607-636 */
static double dgdx_xR0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / dx *
         (-0.5 * p(n, i - 1, j - 1) - 0.5 * p(n, i - 1, j) + 0.5 * p(n, i, j - 1) +
          0.5 * p(n, i, j));
}
/* :671-699 */
static double dgdy_nl_xR0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dy * (-p(n, i, j - 1, dx, dy, gradient_x_x_oneside_R0, gradient_y_interior) +
                     p(n, i, j, dx, dy, gradient_x_x_oneside_R0, gradient_y_interior));
}
/* :733-772 */
static double d2gdx2_xR0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / (dx * dx) *
         (0.5 * p(n, i - 2, j - 1) + 0.5 * p(n, i - 2, j) -
          2.0 * (+0.5 * p(n, i - 1, j - 1) + 0.5 * p(n, i - 1, j)) + 0.5 * p(n, i, j - 1) +
          0.5 * p(n, i, j));
}
/* :809-841 */
static double d2gdxdy_xR0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (p(n, i - 1, j - 1) - p(n, i - 1, j) - p(n, i, j - 1) + p(n, i, j)) * 1.0 / (dx * dy);
}

/* ---------------- y_oneside_L0 (sd_operators_y_oneside_L0_class.f) ---- */
/* :170-196 */
static double dfdx_nl_yL0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dx * (-p(n, i - 1, j, dx, dy, gradient_x_interior, gradient_y_y_oneside_L0) +
                     p(n, i, j, dx, dy, gradient_x_interior, gradient_y_y_oneside_L0));
}
/* :229-258 */
static double dfdy_yL0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / dy *
         (-0.5 * p(n, i - 1, j) - 0.5 * p(n, i, j) + 0.5 * p(n, i - 1, j + 1) +
          0.5 * p(n, i, j + 1));
}
/* :292-331 */
static double d2fdy2_yL0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / (dy * dy) *
         (0.5 * p(n, i - 1, j) + 0.5 * p(n, i, j) -
          2.0 * (+0.5 * p(n, i - 1, j + 1) + 0.5 * p(n, i, j + 1)) + 0.5 * p(n, i - 1, j + 2) +
          0.5 * p(n, i, j + 2));
}
/* :368-400 */
static double d2fdxdy_yL0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (p(n, i - 1, j) - p(n, i, j) - p(n, i - 1, j + 1) + p(n, i, j + 1)) * 1.0 / (dx * dy);
}
/* :428-448 */
static double g_yL0(const ov *n, int i, int j, primary_proc p) {
  return 1.5 * p(n, i, j) - 0.5 * p(n, i, j + 1);
}
/* :481-506 */
static double dgdy_yL0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / dy * (-2.0 * p(n, i, j) + 3.0 * p(n, i, j + 1) - p(n, i, j + 2));
}
/* :542-568 */
static double dgdy_nl_yL0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dy *
         (-2.0 * p(n, i, j, dx, dy, gradient_x_interior, gradient_y_y_oneside_L0) +
          3.0 * p(n, i, j + 1, dx, dy, gradient_x_interior, gradient_y_interior) -
          p(n, i, j + 2, dx, dy, gradient_x_interior, gradient_y_interior));
}
/* :600-629 */
static double dgdx_yL0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / (2.0 * dx) *
         (-1.5 * p(n, i - 1, j) + 0.5 * p(n, i - 1, j + 1) + 1.5 * p(n, i + 1, j) -
          0.5 * p(n, i + 1, j + 1));
}
/* :661-694 */
static double d2gdy2_yL0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 0.5 / (dy * dy) *
         (+3.0 * p(n, i, j) - 5.0 * p(n, i, j + 1) - p(n, i, j + 2) + 5.0 * p(n, i, j + 3) -
          2.0 * p(n, i, j + 4));
}
/* :727-769 */
static double d2gdx2_yL0(const ov *n, int i, int j, primary_proc p, double dx) {
  return (1.0 / (dx * dx)) *
         (1.5 * p(n, i - 1, j) - 0.5 * p(n, i - 1, j + 1) -
          2.0 * (1.5 * p(n, i, j) - 0.5 * p(n, i, j + 1)) + 1.5 * p(n, i + 1, j) -
          0.5 * p(n, i + 1, j + 1));
}
/* :805-839 */
static double d2gdxdy_yL0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (2.0 * p(n, i - 1, j) - 3.0 * p(n, i - 1, j + 1) + p(n, i - 1, j + 2) -
          2.0 * p(n, i + 1, j) + 3.0 * p(n, i + 1, j + 1) - p(n, i + 1, j + 2)) *
         0.5 / (dy * dx);
}

/* ---------------- y_oneside_L1 (sd_operators_y_oneside_L1_class.f) ---- */
/* :160-184 */
static double dgdy_nl_yL1(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dy * (-p(n, i, j - 1, dx, dy, gradient_x_interior, gradient_y_y_oneside_L0) +
                     p(n, i, j, dx, dy, gradient_x_interior, gradient_y_interior));
}
/* :217-249 */
static double d2gdy2_yL1(const ov *n, int i, int j, primary_proc p, double dy) {
  return 0.5 / (dy * dy) *
         (+p(n, i, j - 1) + p(n, i, j) - 7.0 * p(n, i, j + 1) + 7.0 * p(n, i, j + 2) -
          2.0 * p(n, i, j + 3));
}

/* ---------------- y_oneside_R1 (sd_operators_y_oneside_R1_class.f) ---- */
/* :161-185 */
static double dgdy_nl_yR1(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dy * (-p(n, i, j - 1, dx, dy, gradient_x_interior, gradient_y_interior) +
                     p(n, i, j, dx, dy, gradient_x_interior, gradient_y_y_oneside_R0));
}
/* :218-250 */
static double d2gdy2_yR1(const ov *n, int i, int j, primary_proc p, double dy) {
  return 0.5 / (dy * dy) *
         (-2.0 * p(n, i, j - 4) + 7.0 * p(n, i, j - 3) - 7.0 * p(n, i, j - 2) + p(n, i, j - 1) +
          p(n, i, j));
}

/* ---------------- y_oneside_R0 (sd_operators_y_oneside_R0_class.f) ---- */
/* :169-195 */
static double dfdx_nl_yR0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dx * (-p(n, i - 1, j, dx, dy, gradient_x_interior, gradient_y_y_oneside_R0) +
                     p(n, i, j, dx, dy, gradient_x_interior, gradient_y_y_oneside_R0));
}
/* :229-258 */
static double dfdy_yR0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / dy *
         (-0.5 * p(n, i - 1, j - 1) - 0.5 * p(n, i, j - 1) + 0.5 * p(n, i - 1, j) +
          0.5 * p(n, i, j));
}
/* :292-331 */
static double d2fdy2_yR0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / (dy * dy) *
         (0.5 * p(n, i - 1, j - 2) + 0.5 * p(n, i, j - 2) -
          2.0 * (+0.5 * p(n, i - 1, j - 1) + 0.5 * p(n, i, j - 1)) + 0.5 * p(n, i - 1, j) +
          0.5 * p(n, i, j));
}
/* :368-400 */
static double d2fdxdy_yR0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (p(n, i - 1, j - 1) - p(n, i, j - 1) - p(n, i - 1, j) + p(n, i, j)) * 1.0 / (dx * dy);
}
/* :428-448 */
static double g_yR0(const ov *n, int i, int j, primary_proc p) {
  return -0.5 * p(n, i, j - 2) + 1.5 * p(n, i, j - 1);
}
/* :481-506 */
static double dgdy_yR0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 1.0 / dy * (p(n, i, j - 3) - 3.0 * p(n, i, j - 2) + 2.0 * p(n, i, j - 1));
}
/* :542-568 */
static double dgdy_nl_yR0(const ov *n, int i, int j, secondary_proc p, double dx, double dy) {
  return 1.0 / dy *
         (p(n, i, j - 3, dx, dy, gradient_x_interior, gradient_y_interior) -
          3.0 * p(n, i, j - 2, dx, dy, gradient_x_interior, gradient_y_interior) +
          2.0 * p(n, i, j - 1, dx, dy, gradient_x_interior, gradient_y_y_oneside_R0));
}
/* :601-629 */
static double dgdx_yR0(const ov *n, int i, int j, primary_proc p, double dx) {
  return 1.0 / (2.0 * dx) *
         (+0.5 * p(n, i - 1, j - 2) - 1.5 * p(n, i - 1, j - 1) - 0.5 * p(n, i + 1, j - 2) +
          1.5 * p(n, i + 1, j - 1));
}
/* :662-694 */
static double d2gdy2_yR0(const ov *n, int i, int j, primary_proc p, double dy) {
  return 0.5 / (dy * dy) *
         (-2.0 * p(n, i, j - 5) + 5.0 * p(n, i, j - 4) - p(n, i, j - 3) - 5.0 * p(n, i, j - 2) +
          3.0 * p(n, i, j - 1));
}
/* :728-769 */
static double d2gdx2_yR0(const ov *n, int i, int j, primary_proc p, double dx) {
  return (1.0 / (dx * dx)) *
         (-0.5 * p(n, i - 1, j - 2) + 1.5 * p(n, i - 1, j - 1) -
          2.0 * (-0.5 * p(n, i, j - 2) + 1.5 * p(n, i, j - 1)) - 0.5 * p(n, i + 1, j - 2) +
          1.5 * p(n, i + 1, j - 1));
}
/* :806-840 */
static double d2gdxdy_yR0(const ov *n, int i, int j, primary_proc p, double dx, double dy) {
  return (-p(n, i - 1, j - 3) + 3.0 * p(n, i - 1, j - 2) - 2.0 * p(n, i - 1, j - 1) +
          p(n, i + 1, j - 3) - 3.0 * p(n, i + 1, j - 2) + 2.0 * p(n, i + 1, j - 1)) *
         0.5 / (dy * dx);
}

/* sets: interior operators with the overrides above; gx/gy are the
 * gradients the operator test pairs with each set
 * (test_mattsson_operators.f:190-528) */
static sd_ops make(void) { return SD_INTERIOR; }

static sd_ops S[9];
static int S_init = 0;

static void init_sets(void) {
  sd_ops s;
  S[0] = SD_INTERIOR;
  /* 1: x_L0 */
  s = make();
  s.f = f_xL0; s.dfdx = dfdx_xL0; s.dfdx_nl = dfdx_nl_xL0; s.dfdy = dfdy_xL0;
  s.d2fdx2 = d2fdx2_xL0; s.d2fdy2 = d2fdy2_xL0; s.d2fdxdy = d2fdxdy_xL0;
  s.dgdx = dgdx_xL0; s.dgdy_nl = dgdy_nl_xL0; s.d2gdx2 = d2gdx2_xL0; s.d2gdxdy = d2gdxdy_xL0;
  s.gx = gradient_x_x_oneside_L0;
  S[1] = s;
  /* 2: x_L1 */
  s = make();
  s.dfdx_nl = dfdx_nl_xL1; s.d2fdx2 = d2fdx2_xL1;
  S[2] = s;
  /* 3: x_R1 */
  s = make();
  s.dfdx_nl = dfdx_nl_xR1; s.d2fdx2 = d2fdx2_xR1;
  S[3] = s;
  /* 4: x_R0 */
  s = make();
  s.f = f_xR0; s.dfdx = dfdx_xR0; s.dfdx_nl = dfdx_nl_xR0; s.dfdy = dfdy_xR0;
  s.d2fdx2 = d2fdx2_xR0; s.d2fdy2 = d2fdy2_xR0; s.d2fdxdy = d2fdxdy_xR0;
  s.dgdx = dgdx_xR0; s.dgdy_nl = dgdy_nl_xR0; s.d2gdx2 = d2gdx2_xR0; s.d2gdxdy = d2gdxdy_xR0;
  s.gx = gradient_x_x_oneside_R0;
  S[4] = s;
  /* 5: y_L0 */
  s = make();
  s.dfdx_nl = dfdx_nl_yL0; s.dfdy = dfdy_yL0; s.d2fdy2 = d2fdy2_yL0; s.d2fdxdy = d2fdxdy_yL0;
  s.g = g_yL0; s.dgdx = dgdx_yL0; s.dgdy = dgdy_yL0; s.dgdy_nl = dgdy_nl_yL0;
  s.d2gdx2 = d2gdx2_yL0; s.d2gdy2 = d2gdy2_yL0; s.d2gdxdy = d2gdxdy_yL0;
  s.gy = gradient_y_y_oneside_L0;
  S[5] = s;
  /* 6: y_L1 */
  s = make();
  s.dgdy_nl = dgdy_nl_yL1; s.d2gdy2 = d2gdy2_yL1;
  S[6] = s;
  /* 7: y_R1 */
  s = make();
  s.dgdy_nl = dgdy_nl_yR1; s.d2gdy2 = d2gdy2_yR1;
  S[7] = s;
  /* 8: y_R0 */
  s = make();
  s.dfdx_nl = dfdx_nl_yR0; s.dfdy = dfdy_yR0; s.d2fdy2 = d2fdy2_yR0; s.d2fdxdy = d2fdxdy_yR0;
  s.g = g_yR0; s.dgdx = dgdx_yR0; s.dgdy = dgdy_yR0; s.dgdy_nl = dgdy_nl_yR0;
  s.d2gdx2 = d2gdx2_yR0; s.d2gdy2 = d2gdy2_yR0; s.d2gdxdy = d2gdxdy_yR0;
  s.gy = gradient_y_y_oneside_R0;
  S[8] = s;
  S_init = 1;
}

const sd_ops *orc_sd_set(int set) {
  if (!S_init) init_sets();
  if (set < 0 || set > 8) return 0;
  return &S[set];
}
