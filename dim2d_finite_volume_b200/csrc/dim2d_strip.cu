// dim2d_strip.cu -- fused RK3 stage, warp-streaming variant for sm_100a.
//
// Same physics as k_interior (dim2d_interior.cu) -- node quantities, face
// fluxes, divergence, body force, stage update -- organised so that no
// CTA-wide barrier is needed and every face and node quantity is computed
// once:
//   * a warp owns a strip of 30 interior columns (lane = column) and H rows
//     and marches up the strip one row per iteration;
//   * per-warp shared-memory rings hold 3 rows of the input state (rows
//     y..y+2, 34 columns), 3 rows of velocities (y-1..y+1) and 2 rows of
//     the other node quantities (y, y+1) for 32 columns -- one per lane, so
//     the node pass is a single warp pass;
//   * node quantities: u, v, P, Tcl, 1/(3-rho), Tcap, and the node
//     Laplacian and centred gradient of rho.  The face Laplacian and
//     tangential density derivative of the reference's Mattsson stencils
//     are the averages of the two nodes' values (the same sums, regrouped);
//   * iteration y: issue the global loads of row y+3 (prefetch into
//     registers), compute the node quantities of row y+1, then the x-face
//     between columns x-1 and x of row y and the y-face between rows y and
//     y+1 of column x; the right x-face of the cell comes from lane+1 by a
//     shuffle, the bottom y-face is the top face of the previous iteration
//     (kept in registers); update cell (x, y); store the prefetched row
//     into the ring slot of row y.
// Lane 30 evaluates only the x-face its left neighbour needs; lane 31's
// face work repeats lane 30's / 29's (clamped column, result unused).
// Warps are independent (__syncwarp only), so the latency of one warp's
// loads is hidden by the arithmetic of the others.
//
// On a field open on all sides the launch also integrates the ghost cells
// (open_ghost_cell, one thread each): they take the first CTAs of the
// grid, so their long dependent chains start first and overlap the strips.
// Ghost and interior cells read the same input and write disjoint cells.
#include "dim2d_open.cuh"

namespace dim2d {

namespace {

constexpr int SW = 30;  // cells per strip
constexpr int RC = 34;  // state columns in the ring: c0-2 .. c0+31
constexpr int PC = 32;  // node-quantity columns: c0-1 .. c0+30
constexpr int NS = 3;   // state rows (y .. y+2)
constexpr int NUV = 3;  // velocity rows (y-1 .. y+1)
constexpr int NQ = 2;   // rows of the other node quantities (y, y+1)
enum NodeQ : int { Q_P = 0, Q_TCL, Q_CP, Q_TCAP, Q_LAP, Q_GX, Q_GY, NQV };
constexpr int WARP_DOUBLES = NS * 4 * RC + NUV * 2 * PC + NQ * NQV * PC;

// ring slots are selected by row number modulo the ring depth
struct Ring {
  double* st;  // [NS][4][RC]  rho, m_x, m_y, E
  double* uv;  // [NUV][2][PC] u, v
  double* q;   // [NQ][NQV][PC]
  __device__ __forceinline__ double& r(int row, int v, int col) const {
    return st[((row % NS) * 4 + v) * RC + col];
  }
  __device__ __forceinline__ double& u(int row, int c, int col) const {
    return uv[((row % NUV) * 2 + c) * PC + col];
  }
  __device__ __forceinline__ double& n(int row, int c, int col) const {
    return q[((row % NQ) * NQV + c) * PC + col];
  }
};

// global loads of the state row `row` for columns c0-2+lane and c0+30+lane
__device__ __forceinline__ void load_row(const StageArgs& a, int c0, int row, int lane,
                                         double v[2][4]) {
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const int col = lane + 32 * s;
    const int x = c0 - 2 + col;
    v[s][0] = 1.0;  // benign values past the field edge
    v[s][1] = v[s][2] = v[s][3] = 0.0;
    if (col < RC && x < a.f.nx && row < a.f.ny) {
      const size_t o = (size_t)row * a.f.pitch + x;
      v[s][0] = __ldg(a.uin + o);
      v[s][1] = __ldg(a.uin + o + a.f.plane);
      v[s][2] = __ldg(a.uin + o + 2 * a.f.plane);
      v[s][3] = __ldg(a.uin + o + 3 * a.f.plane);
    }
  }
}

__device__ __forceinline__ void store_row(const Ring& R, int row, int lane, const double v[2][4]) {
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const int col = lane + 32 * s;
    if (col < RC) {
#pragma unroll
      for (int q = 0; q < 4; q++) R.r(row, q, col) = v[s][q];
    }
  }
}

// node quantities of row `row`, column c0-1+lane (needs state rows
// row-1..row+1).  Primitives as node_prim() (dim2d_prim_module.f:242-289,
// 425-453, 515-544, 1056-1071) with 1/rho and 1/(3-rho) from one division;
// Tcap = 0.5/rho |grad rho|^2 with centred gradients (:582-613).
__device__ __forceinline__ void node_row(const Ring& R, int row, int lane, double hrdx,
                                         double hrdy, double rdx2, double rdy2,
                                         const DimConst& k) {
  const int pc = lane, rc = lane + 1;
  const double r = R.r(row, 0, rc);
  const double rw = R.r(row, 0, rc - 1), re = R.r(row, 0, rc + 1);
  const double rs = R.r(row - 1, 0, rc), rn = R.r(row + 1, 0, rc);
  const double tm = 3.0 - r;
  const double inv = 1.0 / (r * tm);
  const double ir = tm * inv;
  const double cp = r * inv;
  const double u = R.r(row, 1, rc) * ir, v = R.r(row, 2, rc) * ir;
  const double w = R.r(row, 3, rc) - 0.5 * r * (u * u + v * v) + 3.0 * (r * r);
  const double gx = hrdx * (re - rw), gy = hrdy * (rn - rs);
  R.u(row, 0, pc) = u;
  R.u(row, 1, pc) = v;
  R.n(row, Q_P, pc) = k.c3cv * cp * w - 3.0 * (r * r);
  R.n(row, Q_TCL, pc) = ir * w;
  R.n(row, Q_CP, pc) = cp;
  R.n(row, Q_TCAP, pc) = 0.5 * ir * (gx * gx + gy * gy);
  R.n(row, Q_LAP, pc) = rdx2 * ((rw - 2.0 * r) + re) + rdy2 * ((rs - 2.0 * r) + rn);
  R.n(row, Q_GX, pc) = gx;
  R.n(row, Q_GY, pc) = gy;
}

// x-face between columns x-1 and x of row y, evaluated for column
// c0 + l (l = the lane, clamped to SW)
template <bool WALL>
__device__ __forceinline__ void x_face(const StageArgs& a, const Ring& R, int l, int x, int y,
                                       double F[4]) {
  const DimConst& k = a.k;
  const int rL = l + 1, rR = l + 2;  // state columns of L, R
  const int pL = l, pR = l + 1;      // node-quantity columns
  FaceIn fi;
  fi.ra = R.r(y, 0, rL); fi.rb = R.r(y, 0, rR);
  fi.mna = R.r(y, 1, rL); fi.mnb = R.r(y, 1, rR);
  fi.mta = R.r(y, 2, rL); fi.mtb = R.r(y, 2, rR);
  fi.ea = R.r(y, 3, rL); fi.eb = R.r(y, 3, rR);
  fi.una = R.u(y, 0, pL); fi.unb = R.u(y, 0, pR);
  fi.uta = R.u(y, 1, pL); fi.utb = R.u(y, 1, pR);
  fi.pa = R.n(y, Q_P, pL); fi.pb = R.n(y, Q_P, pR);
  fi.ta = R.n(y, Q_TCL, pL); fi.tb = R.n(y, Q_TCL, pR);
  fi.ca = R.n(y, Q_CP, pL); fi.cb = R.n(y, Q_CP, pR);
  fi.ka = R.n(y, Q_TCAP, pL); fi.kb = R.n(y, Q_TCAP, pR);
  const double rdx = a.rdx, q_rdy = 0.25 * a.rdy;
  fi.drn = rdx * (fi.rb - fi.ra);
  fi.drt = 0.5 * (R.n(y, Q_GY, pL) + R.n(y, Q_GY, pR));
  fi.dunn = rdx * (fi.unb - fi.una);
  fi.dunt = q_rdy * ((R.u(y + 1, 0, pL) + R.u(y + 1, 0, pR)) - (R.u(y - 1, 0, pL) + R.u(y - 1, 0, pR)));
  fi.dutn = rdx * (fi.utb - fi.uta);
  fi.dutt = q_rdy * ((R.u(y + 1, 1, pL) + R.u(y + 1, 1, pR)) - (R.u(y - 1, 1, pL) + R.u(y - 1, 1, pR)));
  fi.lap = 0.5 * (R.n(y, Q_LAP, pL) + R.n(y, Q_LAP, pR));
  fi.dtn = rdx * (fi.tb - fi.ta);
  fi.dkn = rdx * (fi.kb - fi.ka);
  const bool w_face = WALL && a.wall_w && x == BC;
  const bool e_face = WALL && a.wall_e && x == a.f.nx - BC;
  if (w_face || e_face) {
    const int p = w_face ? pR : pL;
    const double tl = k.c38cv * (R.n(y, Q_TCL, p) - k.iwe * R.n(y, Q_TCAP, p));
    const double q = wall_heat_flux(a.wall, a.xmap0 + x * a.dx);
    wall_face_flux(fi, tl, a.dx, q, w_face ? q : -q, k, F);
  } else {
    face_flux(fi, k, F);
  }
}

// y-face between rows yb and yb+1 of column c0 + l (l = the lane, clamped
// to SW-1); output in conservative order (mass, m_x, m_y, E)
template <bool WALL>
__device__ __forceinline__ void y_face(const StageArgs& a, const Ring& R, int l, int x, int yb,
                                       double G[4]) {
  const DimConst& k = a.k;
  const int rc = l + 2, pc = l + 1;
  const int yt = yb + 1;
  FaceIn fi;
  fi.ra = R.r(yb, 0, rc); fi.rb = R.r(yt, 0, rc);
  fi.mna = R.r(yb, 2, rc); fi.mnb = R.r(yt, 2, rc);
  fi.mta = R.r(yb, 1, rc); fi.mtb = R.r(yt, 1, rc);
  fi.ea = R.r(yb, 3, rc); fi.eb = R.r(yt, 3, rc);
  fi.una = R.u(yb, 1, pc); fi.unb = R.u(yt, 1, pc);
  fi.uta = R.u(yb, 0, pc); fi.utb = R.u(yt, 0, pc);
  fi.pa = R.n(yb, Q_P, pc); fi.pb = R.n(yt, Q_P, pc);
  fi.ta = R.n(yb, Q_TCL, pc); fi.tb = R.n(yt, Q_TCL, pc);
  fi.ca = R.n(yb, Q_CP, pc); fi.cb = R.n(yt, Q_CP, pc);
  fi.ka = R.n(yb, Q_TCAP, pc); fi.kb = R.n(yt, Q_TCAP, pc);
  const double rdy = a.rdy, q_rdx = 0.25 * a.rdx;
  fi.drn = rdy * (fi.rb - fi.ra);
  fi.drt = 0.5 * (R.n(yb, Q_GX, pc) + R.n(yt, Q_GX, pc));
  fi.dunn = rdy * (fi.unb - fi.una);
  fi.dunt = q_rdx * ((R.u(yb, 1, pc + 1) + R.u(yt, 1, pc + 1)) - (R.u(yb, 1, pc - 1) + R.u(yt, 1, pc - 1)));
  fi.dutn = rdy * (fi.utb - fi.uta);
  fi.dutt = q_rdx * ((R.u(yb, 0, pc + 1) + R.u(yt, 0, pc + 1)) - (R.u(yb, 0, pc - 1) + R.u(yt, 0, pc - 1)));
  fi.lap = 0.5 * (R.n(yb, Q_LAP, pc) + R.n(yt, Q_LAP, pc));
  fi.dtn = rdy * (fi.tb - fi.ta);
  fi.dkn = rdy * (fi.kb - fi.ka);
  double F[4];
  const bool s_face = WALL && a.wall_s && yt == BC;
  const bool n_face = WALL && a.wall_n && yt == a.f.ny - BC;
  if (s_face || n_face) {
    const int row = s_face ? yt : yb;
    const double tl = k.c38cv * (R.n(row, Q_TCL, pc) - k.iwe * R.n(row, Q_TCAP, pc));
    const double q = wall_heat_flux(a.wall, a.xmap0 + x * a.dx);
    wall_face_flux(fi, tl, a.dy, q, s_face ? q : -q, k, F);
  } else {
    face_flux(fi, k, F);
  }
  G[0] = F[0];
  G[1] = F[2];  // momentum_x is tangential on a y-face
  G[2] = F[1];
  G[3] = F[3];
}

// boundary kinds of the strip kernel
enum StripKind : int { K_PLAIN = 0, K_WALL = 1, K_OPEN = 2 };

// grid: [ghost CTAs (K_OPEN only)] + sx * sy strip CTAs, x fastest
template <int H, int WPC, int MINB, int MODE, int KIND>
__global__ void __launch_bounds__(32 * WPC, MINB) k_strip(StageArgs a, int ghost_ctas, int sx) {
  constexpr bool WALL = KIND == K_WALL;
  int b = blockIdx.x;
  if (KIND == K_OPEN) {
    if (b < ghost_ctas) {
      open_ghost_cell(a, b * (32 * WPC) + threadIdx.x, MODE);
      return;
    }
    b -= ghost_ctas;
  }
  extern __shared__ __align__(16) double sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* base = sm + warp * WARP_DOUBLES;
  const Ring R{base, base + NS * 4 * RC, base + NS * 4 * RC + NUV * 2 * PC};
  const Field f = a.f;
  const int c0 = BC + (b % sx) * SW;
  const int y0 = BC + ((b / sx) * WPC + warp) * H;
  const int ylast = f.ny - BC - 1;
  if (y0 > ylast) return;  // the whole warp leaves; no CTA barrier is used
  const int y1 = min(y0 + H, ylast + 1);
  const int x = c0 + lane;
  const int xl = min(lane, SW), yl = min(lane, SW - 1);  // clamped face columns
  const DimConst& k = a.k;
  const double hrdx = 0.5 * a.rdx, hrdy = 0.5 * a.rdy;
  const double rdx2 = a.rdx * a.rdx, rdy2 = a.rdy * a.rdy;

  // prologue: node quantities of rows y0-1 and y0, bottom face of row y0,
  // state rows y0 .. y0+2 in the ring
  double v[2][4];
#pragma unroll 1
  for (int row = y0 - 2; row <= y0; row++) {
    load_row(a, c0, row, lane, v);
    store_row(R, row, lane, v);
  }
  __syncwarp();
  node_row(R, y0 - 1, lane, hrdx, hrdy, rdx2, rdy2, k);
  load_row(a, c0, y0 + 1, lane, v);
  __syncwarp();  // state row y0-2 is no longer read
  store_row(R, y0 + 1, lane, v);
  __syncwarp();
  node_row(R, y0, lane, hrdx, hrdy, rdx2, rdy2, k);
  __syncwarp();
  double Gb[4];
  y_face<WALL>(a, R, yl, x, y0 - 1, Gb);
  load_row(a, c0, y0 + 2, lane, v);
  __syncwarp();  // state row y0-1 is no longer read
  store_row(R, y0 + 2, lane, v);
  __syncwarp();

  const bool active = lane < SW && x <= f.nx - 1 - BC;
  int ix2 = -1;
  if (a.periodic) {
    const int px = f.nx - 2 * BC;
    if (x < 2 * BC) ix2 = x + px;
    else if (x >= f.nx - 2 * BC) ix2 = x - px;
  }

#pragma unroll 1
  for (int y = y0; y < y1; y++) {
    double nxt[2][4];
    load_row(a, c0, y + 3, lane, nxt);  // prefetch
    node_row(R, y + 1, lane, hrdx, hrdy, rdx2, rdy2, k);
    __syncwarp();
    double Fx[4], Gt[4];
    x_face<WALL>(a, R, xl, x, y, Fx);
    y_face<WALL>(a, R, yl, x, y, Gt);
    double Fr[4];
#pragma unroll
    for (int v = 0; v < 4; v++) Fr[v] = __shfl_down_sync(0xffffffffu, Fx[v], 1);
    if (active) {
      const size_t go = (size_t)y * f.pitch + x;
      int iy2 = -1;
      if (a.periodic) {
        const int py = f.ny - 2 * BC;
        if (y < 2 * BC) iy2 = y + py;
        else if (y >= f.ny - 2 * BC) iy2 = y - py;
      }
      const double uc[4] = {R.r(y, 0, lane + 2), R.r(y, 1, lane + 2), R.r(y, 2, lane + 2),
                            R.r(y, 3, lane + 2)};
#pragma unroll
      for (int v = 0; v < 4; v++) {
        double L = (Fx[v] - Fr[v]) * a.rdx + (Gb[v] - Gt[v]) * a.rdy;
        if (k.gravity_ac) {  // pmodel_eq_class.f:1889-1904
          if (v == 2) L += -uc[0] * k.gravity;
          if (v == 3) L += -uc[2] * k.gravity;
        }
        double out;
        if (MODE == 0) out = L;
        else if (a.stage == 1) out = uc[v] + a.dt * L;
        else out = a.b * __ldg(a.u0 + go + v * f.plane) + (1.0 - a.b) * (uc[v] + a.dt * L);
        double* dst = a.uout + v * f.plane;
        dst[go] = out;
        if (MODE == 1 && a.periodic) {  // periodic_xy/bc_operators_class.f:156-199
          if (ix2 >= 0) dst[(size_t)y * f.pitch + ix2] = out;
          if (iy2 >= 0) {
            dst[(size_t)iy2 * f.pitch + x] = out;
            if (ix2 >= 0) dst[(size_t)iy2 * f.pitch + ix2] = out;
          }
        }
      }
    }
#pragma unroll
    for (int v = 0; v < 4; v++) Gb[v] = Gt[v];
    __syncwarp();  // state row y is no longer read
    store_row(R, y + 3, lane, nxt);
    __syncwarp();
  }
}

template <int H, int WPC, int MINB, int MODE>
const void* strip_fn(int kind) {
  if (kind == K_WALL) return (const void*)k_strip<H, WPC, MINB, MODE, K_WALL>;
  if (kind == K_OPEN) return (const void*)k_strip<H, WPC, MINB, MODE, K_OPEN>;
  return (const void*)k_strip<H, WPC, MINB, MODE, K_PLAIN>;
}

template <int H, int WPC, int MINB>
cudaError_t launch_strip_shape(const StageArgs& a, int mode, cudaStream_t s) {
  const size_t smem = (size_t)WPC * WARP_DOUBLES * sizeof(double);
  const bool wall = a.wall_w || a.wall_e || a.wall_s || a.wall_n;
  const int kind = a.open ? K_OPEN : (wall ? K_WALL : K_PLAIN);
  const void* fn = mode == 0 ? strip_fn<H, WPC, MINB, 0>(kind) : strip_fn<H, WPC, MINB, 1>(kind);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int sx = (a.f.nx - 2 * BC + SW - 1) / SW;
  const int sy = (a.f.ny - 2 * BC + H * WPC - 1) / (H * WPC);
  int ghost_ctas = kind == K_OPEN ? (open_ghost_count(a.f) + 32 * WPC - 1) / (32 * WPC) : 0;
  const unsigned blocks = (unsigned)ghost_ctas + (unsigned)sx * (unsigned)sy;
  StageArgs aa = a;
  void* args[] = {&aa, &ghost_ctas, &sx};
  return cudaLaunchKernel(fn, dim3(blocks), dim3(32 * WPC), args, smem, s);
}

}  // namespace

// shape id -> (rows per warp, warps per CTA, minimum resident CTAs per SM
// requested from the register allocator)
cudaError_t launch_strip_stage(const StageArgs& a, int mode, int shape, cudaStream_t s) {
  switch (shape) {
    case 0: return launch_strip_shape<8, 4, 4>(a, mode, s);
    case 1: return launch_strip_shape<16, 4, 4>(a, mode, s);
    case 2: return launch_strip_shape<16, 4, 5>(a, mode, s);
    case 3: return launch_strip_shape<8, 4, 5>(a, mode, s);
    case 4: return launch_strip_shape<16, 8, 2>(a, mode, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dim2d
