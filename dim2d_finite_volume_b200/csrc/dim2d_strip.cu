// dim2d_strip.cu -- fused RK3 stage, warp-streaming variant for sm_100a.
//
// Same arithmetic as k_interior (dim2d_interior.cu) -- primitives once per
// node, face fluxes, divergence, body force, stage update -- organised so
// that no CTA-wide barrier is needed and every face is computed once:
//   * a warp owns a strip of 31 interior columns (lane = column) and H rows
//     and marches up the strip one row per iteration;
//   * a per-warp shared-memory ring holds 5 rows of the input state
//     (36 columns x 4 variables) and 3 rows of primitives (34 columns);
//   * iteration y: issue the global loads of row y+3 (prefetch into
//     registers), compute the primitives of row y+1, then the x-face
//     between columns x-1 and x of row y and the y-face between rows y and
//     y+1 of column x; the right x-face of the cell comes from lane+1 by a
//     shuffle, the bottom y-face is the top face of the previous iteration
//     (kept in registers); update cell (x, y); store the prefetched row
//     into the ring slot of row y-2.
// Lane 31 computes only the x-face its left neighbour needs.  Warps are
// independent (__syncwarp only), so the latency of one warp's loads is
// hidden by the arithmetic of the others.
//
// On a field open on all sides the launch also integrates the ghost cells
// (open_ghost_cell, one thread each): they take the first CTAs of the
// grid, so their long dependent chains start first and overlap the strips.
// Ghost and interior cells read the same input and write disjoint cells.
#include "dim2d_open.cuh"

namespace dim2d {

namespace {

constexpr int SW = 31;  // cells per strip
constexpr int RC = 36;  // state columns in the ring: c0-2 .. c0+33
constexpr int PC = 34;  // primitive columns: c0-1 .. c0+32
constexpr int RR = 5;   // state rows in the ring
constexpr int PR = 3;   // primitive rows in the ring
constexpr int NPRIM = 6;
constexpr int WARP_DOUBLES = RR * 4 * RC + PR * NPRIM * PC;

struct Ring {
  double* raw;   // [RR][4][RC]
  double* prim;  // [PR][NPRIM][PC]: u, v, p, tcl, cp, tcap
  __device__ __forceinline__ double& r(int row, int v, int col) const {
    return raw[(row % RR) * 4 * RC + v * RC + col];
  }
  __device__ __forceinline__ double& p(int row, int q, int col) const {
    return prim[(row % PR) * NPRIM * PC + q * PC + col];
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

// primitives of ring row `row` (needs state rows row-1..row+1)
__device__ __forceinline__ void prim_row(const Ring& R, int row, int lane, double hrdx,
                                         double hrdy, const DimConst& k) {
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const int pc = lane + 32 * s;
    if (pc < PC) {
      const int rc = pc + 1;
      const double r = R.r(row, 0, rc);
      const NodePrim q = node_prim(r, R.r(row, 1, rc), R.r(row, 2, rc), R.r(row, 3, rc), k);
      R.p(row, 0, pc) = q.u;
      R.p(row, 1, pc) = q.v;
      R.p(row, 2, pc) = q.p;
      R.p(row, 3, pc) = q.tcl;
      R.p(row, 4, pc) = q.cp;
      R.p(row, 5, pc) = node_tcap(r, R.r(row, 0, rc - 1), R.r(row, 0, rc + 1),
                                  R.r(row - 1, 0, rc), R.r(row + 1, 0, rc), hrdx, hrdy);
    }
  }
}

// x-face between columns x-1 and x of row y; lane's column x = c0 + lane
template <bool WALL>
__device__ __forceinline__ void x_face(const StageArgs& a, const Ring& R, int lane, int x, int y,
                                       double F[4]) {
  const DimConst& k = a.k;
  const int rL = lane + 1, rR = lane + 2;  // state columns of L, R
  const int pL = lane, pR = lane + 1;      // primitive columns
  FaceIn fi;
  fi.ra = R.r(y, 0, rL); fi.rb = R.r(y, 0, rR);
  fi.mna = R.r(y, 1, rL); fi.mnb = R.r(y, 1, rR);
  fi.mta = R.r(y, 2, rL); fi.mtb = R.r(y, 2, rR);
  fi.ea = R.r(y, 3, rL); fi.eb = R.r(y, 3, rR);
  fi.una = R.p(y, 0, pL); fi.unb = R.p(y, 0, pR);
  fi.uta = R.p(y, 1, pL); fi.utb = R.p(y, 1, pR);
  fi.pa = R.p(y, 2, pL); fi.pb = R.p(y, 2, pR);
  fi.ta = R.p(y, 3, pL); fi.tb = R.p(y, 3, pR);
  fi.ca = R.p(y, 4, pL); fi.cb = R.p(y, 4, pR);
  fi.ka = R.p(y, 5, pL); fi.kb = R.p(y, 5, pR);
  const double rdx = a.rdx, q_rdy = 0.25 * a.rdy;
  const double rLp = R.r(y + 1, 0, rL), rRp = R.r(y + 1, 0, rR);
  const double rLm = R.r(y - 1, 0, rL), rRm = R.r(y - 1, 0, rR);
  fi.drn = rdx * (fi.rb - fi.ra);
  fi.drt = q_rdy * ((rLp + rRp) - (rLm + rRm));
  fi.dunn = rdx * (fi.unb - fi.una);
  fi.dunt = q_rdy * ((R.p(y + 1, 0, pL) + R.p(y + 1, 0, pR)) - (R.p(y - 1, 0, pL) + R.p(y - 1, 0, pR)));
  fi.dutn = rdx * (fi.utb - fi.uta);
  fi.dutt = q_rdy * ((R.p(y + 1, 1, pL) + R.p(y + 1, 1, pR)) - (R.p(y - 1, 1, pL) + R.p(y - 1, 1, pR)));
  const double d2n = 0.5 * rdx * rdx * (R.r(y, 0, rL - 1) - fi.ra - fi.rb + R.r(y, 0, rR + 1));
  const double d2t = 0.5 * a.rdy * a.rdy * ((rLm + rRm) - 2.0 * (fi.ra + fi.rb) + (rLp + rRp));
  fi.lap = d2n + d2t;
  fi.dtn = rdx * (fi.tb - fi.ta);
  fi.dkn = rdx * (fi.kb - fi.ka);
  const bool w_face = WALL && a.wall_w && x == BC;
  const bool e_face = WALL && a.wall_e && x == a.f.nx - BC;
  if (w_face || e_face) {
    const int p = w_face ? pR : pL;
    const double tl = k.c38cv * (R.p(y, 3, p) - k.iwe * R.p(y, 5, p));
    const double q = wall_heat_flux(a.wall, a.xmap0 + x * a.dx);
    wall_face_flux(fi, tl, a.dx, q, w_face ? q : -q, k, F);
  } else {
    face_flux(fi, k, F);
  }
}

// y-face between rows yb and yb+1 of column x = c0 + lane; output in
// conservative order (mass, m_x, m_y, E)
template <bool WALL>
__device__ __forceinline__ void y_face(const StageArgs& a, const Ring& R, int lane, int x, int yb,
                                       double G[4]) {
  const DimConst& k = a.k;
  const int rc = lane + 2, pc = lane + 1;
  const int yt = yb + 1;
  FaceIn fi;
  fi.ra = R.r(yb, 0, rc); fi.rb = R.r(yt, 0, rc);
  fi.mna = R.r(yb, 2, rc); fi.mnb = R.r(yt, 2, rc);
  fi.mta = R.r(yb, 1, rc); fi.mtb = R.r(yt, 1, rc);
  fi.ea = R.r(yb, 3, rc); fi.eb = R.r(yt, 3, rc);
  fi.una = R.p(yb, 1, pc); fi.unb = R.p(yt, 1, pc);
  fi.uta = R.p(yb, 0, pc); fi.utb = R.p(yt, 0, pc);
  fi.pa = R.p(yb, 2, pc); fi.pb = R.p(yt, 2, pc);
  fi.ta = R.p(yb, 3, pc); fi.tb = R.p(yt, 3, pc);
  fi.ca = R.p(yb, 4, pc); fi.cb = R.p(yt, 4, pc);
  fi.ka = R.p(yb, 5, pc); fi.kb = R.p(yt, 5, pc);
  const double rdy = a.rdy, q_rdx = 0.25 * a.rdx;
  const double rBp = R.r(yb, 0, rc + 1), rTp = R.r(yt, 0, rc + 1);
  const double rBm = R.r(yb, 0, rc - 1), rTm = R.r(yt, 0, rc - 1);
  fi.drn = rdy * (fi.rb - fi.ra);
  fi.drt = q_rdx * ((rBp + rTp) - (rBm + rTm));
  fi.dunn = rdy * (fi.unb - fi.una);
  fi.dunt = q_rdx * ((R.p(yb, 1, pc + 1) + R.p(yt, 1, pc + 1)) - (R.p(yb, 1, pc - 1) + R.p(yt, 1, pc - 1)));
  fi.dutn = rdy * (fi.utb - fi.uta);
  fi.dutt = q_rdx * ((R.p(yb, 0, pc + 1) + R.p(yt, 0, pc + 1)) - (R.p(yb, 0, pc - 1) + R.p(yt, 0, pc - 1)));
  const double d2n = 0.5 * rdy * rdy * (R.r(yb - 1, 0, rc) - fi.ra - fi.rb + R.r(yt + 1, 0, rc));
  const double d2t = 0.5 * a.rdx * a.rdx * ((rBm + rTm) - 2.0 * (fi.ra + fi.rb) + (rBp + rTp));
  fi.lap = d2n + d2t;
  fi.dtn = rdy * (fi.tb - fi.ta);
  fi.dkn = rdy * (fi.kb - fi.ka);
  double F[4];
  const bool s_face = WALL && a.wall_s && yt == BC;
  const bool n_face = WALL && a.wall_n && yt == a.f.ny - BC;
  if (s_face || n_face) {
    const int row = s_face ? yt : yb;
    const double tl = k.c38cv * (R.p(row, 3, pc) - k.iwe * R.p(row, 5, pc));
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
template <int H, int WPC, int MODE, int KIND>
__global__ void __launch_bounds__(32 * WPC) k_strip(StageArgs a, int ghost_ctas, int sx) {
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
  const Ring R{sm + warp * WARP_DOUBLES, sm + warp * WARP_DOUBLES + RR * 4 * RC};
  const Field f = a.f;
  const int c0 = BC + (b % sx) * SW;
  const int y0 = BC + ((b / sx) * WPC + warp) * H;
  const int ylast = f.ny - BC - 1;
  if (y0 > ylast) return;  // the whole warp leaves; no CTA barrier is used
  const int y1 = min(y0 + H, ylast + 1);
  const int x = c0 + lane;
  const DimConst& k = a.k;
  const double hrdx = 0.5 * a.rdx, hrdy = 0.5 * a.rdy;

  // prologue: state rows y0-2 .. y0+2, primitives of rows y0-1 and y0,
  // bottom face of row y0
  {
    double v[2][4];
#pragma unroll 1
    for (int row = y0 - 2; row <= y0 + 2; row++) {
      load_row(a, c0, row, lane, v);
      store_row(R, row, lane, v);
    }
  }
  __syncwarp();
  prim_row(R, y0 - 1, lane, hrdx, hrdy, k);
  prim_row(R, y0, lane, hrdx, hrdy, k);
  __syncwarp();
  double Gb[4];
  y_face<WALL>(a, R, lane, x, y0 - 1, Gb);

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
    prim_row(R, y + 1, lane, hrdx, hrdy, k);
    __syncwarp();
    double Fx[4], Gt[4];
    x_face<WALL>(a, R, lane, x, y, Fx);
    y_face<WALL>(a, R, lane, x, y, Gt);
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
    store_row(R, y + 3, lane, nxt);
    __syncwarp();
  }
}

template <int H, int WPC, int MODE>
const void* strip_fn(int kind) {
  if (kind == K_WALL) return (const void*)k_strip<H, WPC, MODE, K_WALL>;
  if (kind == K_OPEN) return (const void*)k_strip<H, WPC, MODE, K_OPEN>;
  return (const void*)k_strip<H, WPC, MODE, K_PLAIN>;
}

template <int H, int WPC>
cudaError_t launch_strip_shape(const StageArgs& a, int mode, cudaStream_t s) {
  const size_t smem = (size_t)WPC * WARP_DOUBLES * sizeof(double);
  const bool wall = a.wall_w || a.wall_e || a.wall_s || a.wall_n;
  const int kind = a.open ? K_OPEN : (wall ? K_WALL : K_PLAIN);
  const void* fn = mode == 0 ? strip_fn<H, WPC, 0>(kind) : strip_fn<H, WPC, 1>(kind);
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

// shape id: 0 = (H 8, 4 warps), 1 = (16, 4), 2 = (32, 4), 3 = (16, 8), 4 = (8, 8)
cudaError_t launch_strip_stage(const StageArgs& a, int mode, int shape, cudaStream_t s) {
  switch (shape) {
    case 0: return launch_strip_shape<8, 4>(a, mode, s);
    case 1: return launch_strip_shape<16, 4>(a, mode, s);
    case 2: return launch_strip_shape<32, 4>(a, mode, s);
    case 3: return launch_strip_shape<16, 8>(a, mode, s);
    case 4: return launch_strip_shape<8, 8>(a, mode, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dim2d
