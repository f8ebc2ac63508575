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
// On a field with open sections the launch also integrates their ghost
// cells (open_ghost_cell, one thread each): they take the first CTAs of the
// grid, so their long dependent chains start first and overlap the strips.
// Ghost and interior cells read the same input and write disjoint cells.
// the ghost-cell and node-pass code of this file runs inside the persistent
// kernel, whose inputs change during the launch: coherent loads
#define DIM2D_COHERENT_LOADS
#include "dim2d_nodebc.cuh"
#include "dim2d_open.cuh"

namespace dim2d {

namespace {

constexpr int SW = 30;  // cells per strip
constexpr int RC = 34;  // state columns in the ring: c0-2 .. c0+31
constexpr int PC = 34;  // node-quantity columns: c0-1 .. c0+32 (the last two are
                        // padding read only by lane 31, whose faces are unused)
constexpr int NS = 4;   // state rows (y .. y+2, and the row y+3 landing)
constexpr int NUV = 3;  // velocity rows (y-1 .. y+1)
constexpr int NQ = 2;   // rows of the other node quantities (y, y+1)
// node quantities besides u, v; GXH/GYH = half the centred density
// gradient, LAPH = half the density Laplacian
enum NodeQ : int { Q_P = 0, Q_TCL, Q_CP, Q_TCAP, Q_LAPH, Q_GXH, Q_GYH, NQV };
constexpr int ST_ROW = 4 * RC;    // doubles per state row (4 variables)
constexpr int UV_ROW = 2 * PC;    // doubles per velocity row
constexpr int Q_ROW = NQV * PC;   // doubles per node-quantity row
constexpr int UN_ROW = 4 * 32;    // u^n of one row of the strip's cells (4 variables)
constexpr int WARP_DOUBLES = NS * ST_ROW + NUV * UV_ROW + NQ * Q_ROW + 2 * UN_ROW;

extern __shared__ __align__(16) double g_ring[];

// Ring rows are addressed by offsets into g_ring that already include the
// warp's base and the lane's column; the offsets rotate as the warp moves
// up, so every access below is a register plus a compile-time constant.
#define ST(o, v, dc) g_ring[(o) + (v) * RC + (dc)]
#define UV(o, c, dc) g_ring[(o) + (c) * PC + (dc)]
#define NQ_(o, c, dc) g_ring[(o) + (c) * PC + (dc)]

// Asynchronous global -> shared copies (cp.async): the next state row and
// the next row's u^n land in the ring while the warp computes, without
// passing through registers.  Completion is per thread (commit / wait
// groups); a __syncwarp after the wait makes the whole row visible.
__device__ __forceinline__ void cp_async16(double* smem, const double* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
// wait until at most N of this thread's most recent groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A stage launched as a programmatic dependent of the node pass before it
// (StageArgs::node_sides != 0) starts while that pass runs: a warp whose
// rows or columns reach a side the pass writes waits for the pass (and its
// memory) before its first read; the other warps read only cells the
// previous stage wrote, complete before the pass began.
__device__ __forceinline__ void wait_for_node_pass() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
}
// 1 if the warp's reads -- columns c0-2 .. c0+31, rows y0-2 .. y1+2 (the
// last one a prefetch past the strip), clamped to the field -- reach a
// ghost cell of the sides in `sides`
__device__ __forceinline__ bool reads_node_ghosts(int sides, const Field& f, int c0, int y0,
                                                  int y1) {
  return ((sides & NODE_W) && c0 - 2 < BC) || ((sides & NODE_E) && c0 + 31 >= f.nx - BC) ||
         ((sides & NODE_S) && y0 - 2 < BC) || ((sides & NODE_N) && y1 + 2 >= f.ny - BC);
}

// state row `row` into the ring row at offset o (which includes the lane),
// asynchronously: lane p < 17 copies the 16-byte pairs of columns
// c0-2+2p, c0-1+2p of the 4 planes.  Addresses are clamped to the field's
// rows and to its pitch, so no copy leaves the allocation; the clamped
// values land in ring columns that only unused lanes read.  Needs an even
// pitch and 16-byte aligned planes (strip_layout_ok).
__device__ __forceinline__ void async_row(const StageArgs& a, int c0, int row, int lane, int o) {
  if (lane < 17) {
    const int r = min(row, a.f.ny - 1);
    const int xp = min(c0 - 2 + 2 * lane, a.f.pitch - 2);
    const double* src = a.uin + (size_t)r * a.f.pitch + xp;
    double* dst = g_ring + (o - lane) + 2 * lane;
#pragma unroll
    for (int q = 0; q < 4; q++) cp_async16(dst + q * RC, src + q * a.f.plane);
  }
}

// u^n of row y, columns c0 .. c0+31, into the u^n ring row at offset un
// (which includes the lane): lane p < 16 copies the 16-byte pair of columns
// c0+2p, c0+2p+1 of the 4 planes through L2 (cp.async.cg; the persistent
// kernel rereads u^n buffers that other SMs rewrite within its launch, and
// the L2 path is coherent).  Addresses clamped to the pitch like async_row.
__device__ __forceinline__ void async_un(const StageArgs& a, int c0, int y, int un, int lane) {
  if (lane < 16) {
    const int xp = min(c0 + 2 * lane, a.f.pitch - 2);
    const double* src = a.u0 + (size_t)y * a.f.pitch + xp;
    double* dst = g_ring + (un - lane) + 2 * lane;
#pragma unroll
    for (int v = 0; v < 4; v++) cp_async16(dst + v * 32, src + v * a.f.plane);
  }
}

// node quantities of column c0-1+lane of one row: sm/s0/sp = state rows
// below / at / above, ou/oq = output rows.  Primitives as node_prim()
// (dim2d_prim_module.f:242-289, 425-453, 515-544, 1056-1071) with 1/rho
// and 1/(3-rho) from one division; Tcap = 0.5/rho |grad rho|^2 with
// centred gradients (:582-613).
__device__ __forceinline__ void node_row(int sm, int s0, int sp, int ou, int oq, double qrdx,
                                         double qrdy, double hrdx2, double hrdy2,
                                         const DimConst& k) {
  const double r = ST(s0, 0, 1);
  const double rw = ST(s0, 0, 0), re = ST(s0, 0, 2);
  const double rs = ST(sm, 0, 1), rn = ST(sp, 0, 1);
  const double tm = 3.0 - r;
  const double inv = 1.0 / (r * tm);
  const double ir = tm * inv;
  const double cp = r * inv;
  const double u = ST(s0, 1, 1) * ir, v = ST(s0, 2, 1) * ir;
  const double w = ST(s0, 3, 1) - 0.5 * r * (u * u + v * v) + 3.0 * (r * r);
  const double gxh = qrdx * (re - rw), gyh = qrdy * (rn - rs);
  UV(ou, 0, 0) = u;
  UV(ou, 1, 0) = v;
  NQ_(oq, Q_P, 0) = k.c3cv * cp * w - 3.0 * (r * r);
  NQ_(oq, Q_TCL, 0) = ir * w;
  NQ_(oq, Q_CP, 0) = cp;
  NQ_(oq, Q_TCAP, 0) = 2.0 * ir * (gxh * gxh + gyh * gyh);
  NQ_(oq, Q_LAPH, 0) = hrdx2 * ((rw - 2.0 * r) + re) + hrdy2 * ((rs - 2.0 * r) + rn);
  NQ_(oq, Q_GXH, 0) = gxh;
  NQ_(oq, Q_GYH, 0) = gyh;
}

// x-face between columns x-1 and x of row y: s0 = state row y, um/u0/up =
// velocity rows y-1, y, y+1, q0 = node row y
template <bool WALL>
__device__ __forceinline__ void x_face(const StageArgs& a, int s0, int um, int u0, int up, int q0,
                                       int x, double F[4]) {
  const DimConst& k = a.k;
  FaceIn fi;
  fi.ra = ST(s0, 0, 1); fi.rb = ST(s0, 0, 2);
  fi.mna = ST(s0, 1, 1); fi.mnb = ST(s0, 1, 2);
  fi.mta = ST(s0, 2, 1); fi.mtb = ST(s0, 2, 2);
  fi.ea = ST(s0, 3, 1); fi.eb = ST(s0, 3, 2);
  fi.una = UV(u0, 0, 0); fi.unb = UV(u0, 0, 1);
  fi.uta = UV(u0, 1, 0); fi.utb = UV(u0, 1, 1);
  fi.pa = NQ_(q0, Q_P, 0); fi.pb = NQ_(q0, Q_P, 1);
  fi.ta = NQ_(q0, Q_TCL, 0); fi.tb = NQ_(q0, Q_TCL, 1);
  fi.ca = NQ_(q0, Q_CP, 0); fi.cb = NQ_(q0, Q_CP, 1);
  fi.ka = NQ_(q0, Q_TCAP, 0); fi.kb = NQ_(q0, Q_TCAP, 1);
  const double rdx = a.rdx, q_rdy = 0.25 * a.rdy;
  fi.drn = rdx * (fi.rb - fi.ra);
  fi.drt = NQ_(q0, Q_GYH, 0) + NQ_(q0, Q_GYH, 1);
  fi.dunn = rdx * (fi.unb - fi.una);
  fi.dunt = q_rdy * ((UV(up, 0, 0) + UV(up, 0, 1)) - (UV(um, 0, 0) + UV(um, 0, 1)));
  fi.dutn = rdx * (fi.utb - fi.uta);
  fi.dutt = q_rdy * ((UV(up, 1, 0) + UV(up, 1, 1)) - (UV(um, 1, 0) + UV(um, 1, 1)));
  fi.lap = NQ_(q0, Q_LAPH, 0) + NQ_(q0, Q_LAPH, 1);
  fi.dtn = rdx * (fi.tb - fi.ta);
  fi.dkn = rdx * (fi.kb - fi.ka);
  const bool w_face = WALL && a.wall_w && x == BC;
  const bool e_face = WALL && a.wall_e && x == a.f.nx - BC;
  if (w_face || e_face) {
    const int dc = w_face ? 1 : 0;
    const double tl = k.c38cv * (NQ_(q0, Q_TCL, dc) - k.iwe * NQ_(q0, Q_TCAP, dc));
    const double q = wall_heat_flux(a.wall, a.xmap0 + x * a.dx);
    wall_face_flux(fi, tl, a.dx, q, w_face ? q : -q, k, F);
  } else {
    face_flux(fi, k, F);
  }
}

// y-face between rows yb and yb+1 of column x: sb/st = state rows yb, yb+1,
// ub/ut = velocity rows, qb/qt = node rows; output in conservative order
// (mass, m_x, m_y, E)
template <bool WALL>
__device__ __forceinline__ void y_face(const StageArgs& a, int sb, int st, int ub, int ut, int qb,
                                       int qt, int x, int yb, double G[4]) {
  const DimConst& k = a.k;
  const int yt = yb + 1;
  FaceIn fi;
  fi.ra = ST(sb, 0, 2); fi.rb = ST(st, 0, 2);
  fi.mna = ST(sb, 2, 2); fi.mnb = ST(st, 2, 2);
  fi.mta = ST(sb, 1, 2); fi.mtb = ST(st, 1, 2);
  fi.ea = ST(sb, 3, 2); fi.eb = ST(st, 3, 2);
  fi.una = UV(ub, 1, 1); fi.unb = UV(ut, 1, 1);
  fi.uta = UV(ub, 0, 1); fi.utb = UV(ut, 0, 1);
  fi.pa = NQ_(qb, Q_P, 1); fi.pb = NQ_(qt, Q_P, 1);
  fi.ta = NQ_(qb, Q_TCL, 1); fi.tb = NQ_(qt, Q_TCL, 1);
  fi.ca = NQ_(qb, Q_CP, 1); fi.cb = NQ_(qt, Q_CP, 1);
  fi.ka = NQ_(qb, Q_TCAP, 1); fi.kb = NQ_(qt, Q_TCAP, 1);
  const double rdy = a.rdy, q_rdx = 0.25 * a.rdx;
  fi.drn = rdy * (fi.rb - fi.ra);
  fi.drt = NQ_(qb, Q_GXH, 1) + NQ_(qt, Q_GXH, 1);
  fi.dunn = rdy * (fi.unb - fi.una);
  fi.dunt = q_rdx * ((UV(ub, 1, 2) + UV(ut, 1, 2)) - (UV(ub, 1, 0) + UV(ut, 1, 0)));
  fi.dutn = rdy * (fi.utb - fi.uta);
  fi.dutt = q_rdx * ((UV(ub, 0, 2) + UV(ut, 0, 2)) - (UV(ub, 0, 0) + UV(ut, 0, 0)));
  fi.lap = NQ_(qb, Q_LAPH, 1) + NQ_(qt, Q_LAPH, 1);
  fi.dtn = rdy * (fi.tb - fi.ta);
  fi.dkn = rdy * (fi.kb - fi.ka);
  double F[4];
  const bool s_face = WALL && a.wall_s && yt == BC;
  const bool n_face = WALL && a.wall_n && yt == a.f.ny - BC;
  if (s_face || n_face) {
    const int qo = s_face ? qt : qb;
    const double tl = k.c38cv * (NQ_(qo, Q_TCL, 1) - k.iwe * NQ_(qo, Q_TCAP, 1));
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

// ---- mixed precision (DIM2D_MIXED) -----------------------------------
// The node pass runs in FP64 -- the van der Waals inversion for u, v, P,
// Tcl, 1/(3-rho) and Tcap -- and stores FP32 copies of rho, m_x, m_y, E
// and of those quantities; the face pass (stencils and flux formulas)
// reads the FP32 copies and runs in FP32.  Tcap stays FP64 and its normal
// derivative, the third-derivative capillary term of the energy flux, is
// added to the face's energy flux in FP64.  Divergence and RK update are
// FP64 on the FP64 state.
enum NodeF : int {
  F_R = 0, F_MX, F_MY, F_E, F_U, F_V, F_P, F_TCL, F_CP, F_LAPH, F_GXH, F_GYH, NQF
};
constexpr int NM = 3;              // node rows (y-1 .. y+1)
constexpr int F_ROW = NQF * PC;    // floats per node row
// Mixed precision keeps one u^n row (FP64 keeps two, alternating): the next
// row's u^n is copied once the update has read this one, in its own
// cp.async group, and waited for just before the next update.  10.8 KB per
// warp then fits 20 warps per SM (shape 16x4x5, 96 registers).
constexpr int WARP_DOUBLES_MIX = NS * ST_ROW + NM * PC + (NM * F_ROW + 1) / 2 + UN_ROW;
#define FQ(o, c, dc) reinterpret_cast<float*>(g_ring)[(o) + (c) * PC + (dc)]
#define KQ(o, dc) g_ring[(o) + (dc)]

// node quantities of column c0-1+lane of one row (as node_row) into the
// float row fo and the FP64 Tcap row ko
__device__ __forceinline__ void node_row_mix(int sm, int s0, int sp, int fo, int ko, double qrdx,
                                             double qrdy, double hrdx2, double hrdy2,
                                             const DimConst& k) {
  const double r = ST(s0, 0, 1);
  const double rw = ST(s0, 0, 0), re = ST(s0, 0, 2);
  const double rs = ST(sm, 0, 1), rn = ST(sp, 0, 1);
  const double mx = ST(s0, 1, 1), my = ST(s0, 2, 1), e = ST(s0, 3, 1);
  const double tm = 3.0 - r;
  const double inv = 1.0 / (r * tm);
  const double ir = tm * inv;
  const double cp = r * inv;
  const double u = mx * ir, v = my * ir;
  const double w = e - 0.5 * r * (u * u + v * v) + 3.0 * (r * r);
  const double gxh = qrdx * (re - rw), gyh = qrdy * (rn - rs);
  FQ(fo, F_R, 0) = (float)r;
  FQ(fo, F_MX, 0) = (float)mx;
  FQ(fo, F_MY, 0) = (float)my;
  FQ(fo, F_E, 0) = (float)e;
  FQ(fo, F_U, 0) = (float)u;
  FQ(fo, F_V, 0) = (float)v;
  FQ(fo, F_P, 0) = (float)(k.c3cv * cp * w - 3.0 * (r * r));
  FQ(fo, F_TCL, 0) = (float)(ir * w);
  FQ(fo, F_CP, 0) = (float)cp;
  FQ(fo, F_LAPH, 0) = (float)(hrdx2 * ((rw - 2.0 * r) + re) + hrdy2 * ((rs - 2.0 * r) + rn));
  FQ(fo, F_GXH, 0) = (float)gxh;
  FQ(fo, F_GYH, 0) = (float)gyh;
  KQ(ko, 0) = 2.0 * ir * (gxh * gxh + gyh * gyh);
}

// FP64 face inputs a wall face flux reads, from the FP32 face inputs
__device__ __forceinline__ FaceIn wall_face_in(const FaceInT<float>& fi) {
  FaceIn d{};
  d.ra = fi.ra;
  d.rb = fi.rb;
  d.drn = fi.drn;
  d.drt = fi.drt;
  d.dutn = fi.dutn;
  d.lap = fi.lap;
  return d;
}

// x-face between columns x-1 and x of row y: fm/f0/fp = node rows y-1, y,
// y+1, k0 = Tcap row y
template <bool WALL>
__device__ __forceinline__ void x_face_mix(const StageArgs& a, const FluxCoefF& kf, int fm, int f0,
                                           int fp, int k0, int x, double F[4]) {
  const DimConst& k = a.k;
  FaceInT<float> fi;
  fi.ra = FQ(f0, F_R, 0); fi.rb = FQ(f0, F_R, 1);
  fi.mna = FQ(f0, F_MX, 0); fi.mnb = FQ(f0, F_MX, 1);
  fi.mta = FQ(f0, F_MY, 0); fi.mtb = FQ(f0, F_MY, 1);
  fi.ea = FQ(f0, F_E, 0); fi.eb = FQ(f0, F_E, 1);
  fi.una = FQ(f0, F_U, 0); fi.unb = FQ(f0, F_U, 1);
  fi.uta = FQ(f0, F_V, 0); fi.utb = FQ(f0, F_V, 1);
  fi.pa = FQ(f0, F_P, 0); fi.pb = FQ(f0, F_P, 1);
  fi.ta = FQ(f0, F_TCL, 0); fi.tb = FQ(f0, F_TCL, 1);
  fi.ca = FQ(f0, F_CP, 0); fi.cb = FQ(f0, F_CP, 1);
  fi.ka = fi.kb = 0.0f;
  const float rdx = (float)a.rdx, q_rdy = 0.25f * (float)a.rdy;
  fi.drn = rdx * (fi.rb - fi.ra);
  fi.drt = FQ(f0, F_GYH, 0) + FQ(f0, F_GYH, 1);
  fi.dunn = rdx * (fi.unb - fi.una);
  fi.dunt = q_rdy * ((FQ(fp, F_U, 0) + FQ(fp, F_U, 1)) - (FQ(fm, F_U, 0) + FQ(fm, F_U, 1)));
  fi.dutn = rdx * (fi.utb - fi.uta);
  fi.dutt = q_rdy * ((FQ(fp, F_V, 0) + FQ(fp, F_V, 1)) - (FQ(fm, F_V, 0) + FQ(fm, F_V, 1)));
  fi.lap = FQ(f0, F_LAPH, 0) + FQ(f0, F_LAPH, 1);
  fi.dtn = rdx * (fi.tb - fi.ta);
  fi.dkn = 0.0f;
  const bool w_face = WALL && a.wall_w && x == BC;
  const bool e_face = WALL && a.wall_e && x == a.f.nx - BC;
  if (w_face || e_face) {
    const int dc = w_face ? 1 : 0;
    const double tl = k.c38cv * ((double)FQ(f0, F_TCL, dc) - k.iwe * KQ(k0, dc));
    const double q = wall_heat_flux(a.wall, a.xmap0 + x * a.dx);
    wall_face_flux(wall_face_in(fi), tl, a.dx, q, w_face ? q : -q, k, F);
    return;
  }
  float Ff[4];
  face_flux_t<float, FluxCoefF, false>(fi, kf, Ff);
#pragma unroll
  for (int v = 0; v < 4; v++) F[v] = (double)Ff[v];
  // -(1/We) * (-(1/(Re Pr)) dTcap/dn), FP64
  F[3] += k.iwe * k.irepr * (a.rdx * (KQ(k0, 1) - KQ(k0, 0)));
}

// y-face between rows yb and yb+1 of column x: fb/ft = node rows yb, yb+1,
// kb/kt = their Tcap rows; output in conservative order
template <bool WALL>
__device__ __forceinline__ void y_face_mix(const StageArgs& a, const FluxCoefF& kf, int fb, int ft,
                                           int kb, int kt, int x, int yb, double G[4]) {
  const DimConst& k = a.k;
  const int yt = yb + 1;
  FaceInT<float> fi;
  fi.ra = FQ(fb, F_R, 1); fi.rb = FQ(ft, F_R, 1);
  fi.mna = FQ(fb, F_MY, 1); fi.mnb = FQ(ft, F_MY, 1);
  fi.mta = FQ(fb, F_MX, 1); fi.mtb = FQ(ft, F_MX, 1);
  fi.ea = FQ(fb, F_E, 1); fi.eb = FQ(ft, F_E, 1);
  fi.una = FQ(fb, F_V, 1); fi.unb = FQ(ft, F_V, 1);
  fi.uta = FQ(fb, F_U, 1); fi.utb = FQ(ft, F_U, 1);
  fi.pa = FQ(fb, F_P, 1); fi.pb = FQ(ft, F_P, 1);
  fi.ta = FQ(fb, F_TCL, 1); fi.tb = FQ(ft, F_TCL, 1);
  fi.ca = FQ(fb, F_CP, 1); fi.cb = FQ(ft, F_CP, 1);
  fi.ka = fi.kb = 0.0f;
  const float rdy = (float)a.rdy, q_rdx = 0.25f * (float)a.rdx;
  fi.drn = rdy * (fi.rb - fi.ra);
  fi.drt = FQ(fb, F_GXH, 1) + FQ(ft, F_GXH, 1);
  fi.dunn = rdy * (fi.unb - fi.una);
  fi.dunt = q_rdx * ((FQ(fb, F_V, 2) + FQ(ft, F_V, 2)) - (FQ(fb, F_V, 0) + FQ(ft, F_V, 0)));
  fi.dutn = rdy * (fi.utb - fi.uta);
  fi.dutt = q_rdx * ((FQ(fb, F_U, 2) + FQ(ft, F_U, 2)) - (FQ(fb, F_U, 0) + FQ(ft, F_U, 0)));
  fi.lap = FQ(fb, F_LAPH, 1) + FQ(ft, F_LAPH, 1);
  fi.dtn = rdy * (fi.tb - fi.ta);
  fi.dkn = 0.0f;
  double F[4];
  const bool s_face = WALL && a.wall_s && yt == BC;
  const bool n_face = WALL && a.wall_n && yt == a.f.ny - BC;
  if (s_face || n_face) {
    const int fo = s_face ? ft : fb, ko = s_face ? kt : kb;
    const double tl = k.c38cv * ((double)FQ(fo, F_TCL, 1) - k.iwe * KQ(ko, 1));
    const double q = wall_heat_flux(a.wall, a.xmap0 + x * a.dx);
    wall_face_flux(wall_face_in(fi), tl, a.dy, q, s_face ? q : -q, k, F);
  } else {
    float Ff[4];
    face_flux_t<float, FluxCoefF, false>(fi, kf, Ff);
#pragma unroll
    for (int v = 0; v < 4; v++) F[v] = (double)Ff[v];
    F[3] += k.iwe * k.irepr * (a.rdy * (KQ(kt, 1) - KQ(kb, 1)));
  }
  G[0] = F[0];
  G[1] = F[2];
  G[2] = F[1];
  G[3] = F[3];
}

// boundary kinds of the strip kernel
// K_WALL_OPEN: open sections and a south wall (wall_S_open,
// half_wall_S_open): ghost CTAs of the open sections, wall faces in the strips
enum StripKind : int { K_PLAIN = 0, K_WALL = 1, K_OPEN = 2, K_WALL_OPEN = 3 };

// The strip of one warp: columns c0 .. c0+29 (interior ones), rows y0 ..
// y1-1, with ring slot `warp` of the CTA's shared memory.
template <int MODE, bool WALL, bool MIX>
__device__ __forceinline__ void strip_warp(const StageArgs& a, int c0, int y0, int y1, int warp) {
  const int lane = threadIdx.x & 31;
  const Field f = a.f;
  const int x = c0 + lane;
  const DimConst& k = a.k;
  const double qrdx = 0.25 * a.rdx, qrdy = 0.25 * a.rdy;
  const double hrdx2 = 0.5 * a.rdx * a.rdx, hrdy2 = 0.5 * a.rdy * a.rdy;
  const bool need_un = MODE == 1 && a.stage != 1;

  // ring row offsets (warp base + lane column)
  const int wbase = warp * (MIX ? WARP_DOUBLES_MIX : WARP_DOUBLES);
  const int wb = wbase + lane;
  int s0 = wb, s1 = wb + ST_ROW, s2 = wb + 2 * ST_ROW, s3 = wb + 3 * ST_ROW;  // state rows
  const int ub = wb + NS * ST_ROW;
  int um = ub, u0 = ub + UV_ROW, u1 = ub + 2 * UV_ROW;  // velocity rows
  const int qbase = ub + NUV * UV_ROW;
  int q0 = qbase, q1 = qbase + Q_ROW;                   // node rows
  // mixed precision: Tcap rows (doubles) and FP32 node rows (floats)
  int km = ub, k0 = ub + PC, k1 = ub + 2 * PC;
  const int fbase = 2 * (wbase + NS * ST_ROW + NM * PC) + lane;
  int fm = fbase, f0 = fbase + F_ROW, f1 = fbase + 2 * F_ROW;
  const FluxCoefF kf = flux_coef_f32(k);
  // u^n rows (two, alternating), after the rest of the warp's region
  const int unb = wbase + (MIX ? NS * ST_ROW + NM * PC + (NM * F_ROW + 1) / 2
                               : NS * ST_ROW + NUV * UV_ROW + NQ * Q_ROW) + lane;
  int un0 = unb, un1 = MIX ? unb : unb + UN_ROW;

  if (a.node_sides && reads_node_ghosts(a.node_sides, f, c0, y0, y1)) wait_for_node_pass();

  // prologue: state rows y0-2, y0-1, y0, y0+1 (s3, s2, s0, s1), all four
  // copies in flight together; node quantities of rows y0-1 (um, q1) and
  // y0 (u0, q0); bottom face of row y0; then row y0+2 (into s2) and u^n of
  // row y0 on their way
  async_row(a, c0, y0 - 2, lane, s3);
  async_row(a, c0, y0 - 1, lane, s2);
  async_row(a, c0, y0, lane, s0);
  async_row(a, c0, y0 + 1, lane, s1);
  cp_async_commit();
  cp_async_wait<0>();
  __syncwarp();
  if (MIX) {
    node_row_mix(s3, s2, s0, fm, km, qrdx, qrdy, hrdx2, hrdy2, k);
    node_row_mix(s2, s0, s1, f0, k0, qrdx, qrdy, hrdx2, hrdy2, k);
  } else {
    node_row(s3, s2, s0, um, q1, qrdx, qrdy, hrdx2, hrdy2, k);
    node_row(s2, s0, s1, u0, q0, qrdx, qrdy, hrdx2, hrdy2, k);
  }
  __syncwarp();
  double Gb[4];
  if (MIX) y_face_mix<WALL>(a, kf, fm, f0, km, k0, x, y0 - 1, Gb);
  else y_face<WALL>(a, s2, s0, um, u0, q1, q0, x, y0 - 1, Gb);
  __syncwarp();  // rows y0-2 and y0-1 are no longer read
  async_row(a, c0, y0 + 2, lane, s2);
  if (MIX) cp_async_commit();  // mixed: u^n rows travel in their own groups
  if (need_un) async_un(a, c0, y0, un0, lane);
  cp_async_commit();

  const bool active = lane < SW && x <= f.nx - 1 - BC &&
                      (MODE != 2 || (x >= a.box_x0 && x <= a.box_x1));
  int ix2 = -1;
  if (a.periodic) {
    const int px = f.nx - 2 * BC;
    if (x < 2 * BC) ix2 = x + px;
    else if (x >= f.nx - 2 * BC) ix2 = x - px;
  }

  // s0/s1/s2 = state rows y, y+1, y+2 (row y+2 may still be landing), s3
  // the free slot; un0 = u^n of row y (may be landing), un1 free; um/u0 =
  // velocity rows y-1, y and u1 free; q0 = node row y and q1 free
#pragma unroll 1
  for (int y = y0; y < y1; y++) {
    async_row(a, c0, y + 3, lane, s3);  // next row: lands during this one
    if (!MIX && need_un) async_un(a, c0, y + 1, un1, lane);
    cp_async_commit();
    // FP64: all but the group just issued (rows y+2, u^n(y)); mixed: all
    // but that one and u^n(y)'s, which is waited for before the update
    if (MIX) cp_async_wait<2>();
    else cp_async_wait<1>();
    __syncwarp();
    if (MIX) node_row_mix(s0, s1, s2, f1, k1, qrdx, qrdy, hrdx2, hrdy2, k);
    else node_row(s0, s1, s2, u1, q1, qrdx, qrdy, hrdx2, hrdy2, k);
    __syncwarp();
    double Fx[4], Gt[4];
    if (MIX) {
      x_face_mix<WALL>(a, kf, fm, f0, f1, k0, x, Fx);
      y_face_mix<WALL>(a, kf, f0, f1, k0, k1, x, y, Gt);
    } else {
      x_face<WALL>(a, s0, um, u0, u1, q0, x, Fx);
      y_face<WALL>(a, s0, s1, u0, u1, q0, q1, x, y, Gt);
    }
    double Fr[4];
#pragma unroll
    for (int v = 0; v < 4; v++) Fr[v] = __shfl_down_sync(0xffffffffu, Fx[v], 1);
    if (MIX) {
      cp_async_wait<1>();  // u^n(y)
      __syncwarp();
    }
    {
      // every lane evaluates the update; only active lanes store
      const size_t go = (size_t)y * f.pitch + min(x, f.nx - 1 - BC);
      const double uc[4] = {ST(s0, 0, 2), ST(s0, 1, 2), ST(s0, 2, 2), ST(s0, 3, 2)};
      double out[4];
#pragma unroll
      for (int v = 0; v < 4; v++) {
        double L = (Fx[v] - Fr[v]) * a.rdx + (Gb[v] - Gt[v]) * a.rdy;
        if (k.gravity_ac) {  // pmodel_eq_class.f:1889-1904
          if (v == 2) L += -uc[0] * k.gravity;
          if (v == 3) L += -uc[2] * k.gravity;
        }
        if (MODE != 1) out[v] = L;
        else if (a.stage == 1) out[v] = uc[v] + a.dt * L;
        else out[v] = a.b * g_ring[un0 + v * 32] + (1.0 - a.b) * (uc[v] + a.dt * L);
      }
      // MODE 2 writes the interior_pt points of the layer map only
      if (active && (MODE != 2 || __ldg(a.mask + go) == 1)) {
#pragma unroll
        for (int v = 0; v < 4; v++) a.uout[go + v * f.plane] = out[v];
        if (MODE == 1 && a.periodic) {  // periodic_xy/bc_operators_class.f:156-199
          int iy2 = -1;
          const int py = f.ny - 2 * BC;
          if (y < 2 * BC) iy2 = y + py;
          else if (y >= f.ny - 2 * BC) iy2 = y - py;
#pragma unroll
          for (int v = 0; v < 4; v++) {
            double* dst = a.uout + v * f.plane;
            if (ix2 >= 0) dst[(size_t)y * f.pitch + ix2] = out[v];
            if (iy2 >= 0) {
              dst[(size_t)iy2 * f.pitch + x] = out[v];
              if (ix2 >= 0) dst[(size_t)iy2 * f.pitch + ix2] = out[v];
            }
          }
        }
      }
    }
#pragma unroll
    for (int v = 0; v < 4; v++) Gb[v] = Gt[v];
    __syncwarp();  // row y and u^n(y) are no longer read
    if (MIX) {  // mixed: one u^n slot, refilled now that row y is done
      if (need_un) async_un(a, c0, y + 1, un0, lane);
      cp_async_commit();
    }
    const int t = s0;
    s0 = s1;
    s1 = s2;
    s2 = s3;
    s3 = t;
    const int tn = un0;
    un0 = un1;
    un1 = tn;
    const int tu = um;
    um = u0;
    u0 = u1;
    u1 = tu;
    const int tq = q0;
    q0 = q1;
    q1 = tq;
    const int tf = fm;
    fm = f0;
    f0 = f1;
    f1 = tf;
    const int tk = km;
    km = k0;
    k0 = k1;
    k1 = tk;
  }
  cp_async_wait<0>();  // the copies of rows past the strip land before the warp exits
}

// grid: [ghost CTAs (K_OPEN only)] + sx * sy strip CTAs, x fastest
// The work of strip CTA number b of one field (sx strips per row band).
template <int H, int WPC, int MODE, bool WALL, bool MIX>
__device__ __forceinline__ void strip_cta(const StageArgs& a, int b, int sx) {
  const int warp = threadIdx.x >> 5;
  // MODE 2 (buffer-layer grid): strips over the border box, the first one
  // starting at an even column so that the rows' 16-byte pairs stay aligned
  const int c0 = (MODE == 2 ? (a.box_x0 & ~1) : BC) + (b % sx) * SW;
  const int y0 = (MODE == 2 ? a.box_y0 : BC) + ((b / sx) * WPC + warp) * H;
  const int ylast = MODE == 2 ? a.box_y1 : a.f.ny - BC - 1;
  if (y0 > ylast) return;  // the whole warp leaves; no CTA barrier is used
  strip_warp<MODE, WALL, MIX>(a, c0, y0, min(y0 + H, ylast + 1), warp);
}

template <int H, int WPC, int MINB, int MODE, int KIND, bool MIX>
__global__ void __launch_bounds__(32 * WPC, MINB) k_strip(StageArgs a, int ghost_ctas, int sx) {
  int b = blockIdx.x;
  if (KIND == K_OPEN || KIND == K_WALL_OPEN) {
    if (b < ghost_ctas) {
      if (a.node_sides) wait_for_node_pass();  // ghost frames reach the wall rows
      open_ghost_cell(a, b * (32 * WPC) + threadIdx.x, MODE);
      return;
    }
    b -= ghost_ctas;
  }
  strip_cta<H, WPC, MODE, KIND == K_WALL || KIND == K_WALL_OPEN, MIX>(a, b, sx);
}

// stage arguments of domain i of a batched launch
__device__ __forceinline__ StageArgs batch_stage_args(const BatchStageArgs& P, int i) {
  const BatchDomain& d = P.d[i];
  StageArgs a;
  a.uin = d.uin;
  a.u0 = d.u0;
  a.uout = d.uout;
  a.f = d.f;
  a.dx = d.dx;
  a.dy = d.dy;
  a.rdx = d.rdx;
  a.rdy = d.rdy;
  a.dt = d.dt;
  a.b = P.b;
  a.stage = P.stage;
  a.periodic = d.periodic;
  a.wall_w = a.wall_e = a.wall_n = 0;
  a.wall_s = d.wall_s;
  a.variant = 0;
  a.open = d.open;
  a.node_sides = d.node_sides;
  a.mixed = 0;
  a.t = 0.0;
  a.xmap0 = d.xmap0;
  a.ymap0 = 0.0;
  a.wall = P.wall;
  a.k = P.k;
  return a;
}

// last domain i in [0, n) whose first CTA (ghost0 or strip0) is <= b
template <bool GHOST>
__device__ __forceinline__ int batch_domain(const BatchStageArgs& P, int b) {
  int lo = 0, hi = P.ndom - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    const int first = GHOST ? P.d[mid].ghost0 : P.d[mid].strip0;
    if (first <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// One RK stage of every domain of a batch (one boundary kind): the ghost
// CTAs of all domains first (open and wall kinds: each domain's open
// sections), then every domain's strip CTAs.
template <int H, int WPC, int MINB, int KIND, bool MIX>
__global__ void __launch_bounds__(32 * WPC, MINB)
    k_strip_batch(const __grid_constant__ BatchStageArgs P) {
  int b = blockIdx.x;
  if (KIND == K_OPEN || KIND == K_WALL_OPEN) {
    if (b < P.ghost_ctas) {
      const int i = batch_domain<true>(P, b);
      const StageArgs a = batch_stage_args(P, i);
      if (a.node_sides) wait_for_node_pass();
      open_ghost_cell(a, (b - P.d[i].ghost0) * (32 * WPC) + threadIdx.x, 1);
      return;
    }
    b -= P.ghost_ctas;
  }
  const int i = batch_domain<false>(P, b);
  const StageArgs a = batch_stage_args(P, i);
  strip_cta<H, WPC, 1, KIND == K_WALL || KIND == K_WALL_OPEN, MIX>(a, b - P.d[i].strip0,
                                                                     P.d[i].sx);
}

// ---- persistent batched kernel -----------------------------------------
// Item it of a launch is item it % items_per_step of the per-step table, in
// step it / items_per_step.  Buffer roles of step k (A = buf[0] holds u^n at
// launch, B = buf[1]): u^n = A on even steps and B on odd steps, the other
// one of the pair takes stages 1 and 3, C takes stage 2 -- the A/B swap of
// rk3_step, step after step.
constexpr int PW = 2;  // warps per CTA of the persistent kernel

__device__ __forceinline__ unsigned long long load_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long load_relaxed(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acquire() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// wait until done >= target (every lane loads with acquire semantics);
// false if the launch was stopped or the wait ran out (which stops it)
__device__ bool wait_done(const PersistArgs& P, const unsigned long long* done,
                          unsigned long long target) {
  if (load_acquire(done) >= target) return true;
  const unsigned long long t0 = global_ns();
  unsigned ns = 64;
  // the iteration cap (a few seconds of 2 us sleeps) bounds the wait even
  // if the timer stalled
  for (int it = 0; it < (1 << 21); it++) {
    __nanosleep(ns);
    if (ns < 2048) ns *= 2;
    if (load_acquire(done) >= target) return true;
    if (*(volatile unsigned int*)&P.ctl[0]) return false;
    if (global_ns() - t0 > P.wait_ns) break;
  }
  atomicOr(&P.ctl[1], 1u);
  atomicExch(&P.ctl[0], 1u);
  return false;
}

__device__ __forceinline__ StageArgs persist_stage_args(const PersistArgs& P, const PDomain& d,
                                                        int step, int st) {
  const int odd = (P.step0 + step) & 1;
  double* X = odd ? d.buf[1] : d.buf[0];  // u^n
  double* Y = odd ? d.buf[0] : d.buf[1];
  StageArgs a;
  a.uin = st == 1 ? X : (st == 2 ? Y : d.buf[2]);
  a.u0 = X;
  a.uout = st == 2 ? d.buf[2] : Y;
  a.f = d.f;
  a.dx = d.dx;
  a.dy = d.dy;
  a.rdx = d.rdx;
  a.rdy = d.rdy;
  a.dt = d.dt * P.dt_scale;
  a.b = st == 2 ? 0.75 : (st == 3 ? 1.0 / 3.0 : 0.0);  // rk3tvd_steps_module.f:225,444
  a.stage = st;
  a.periodic = d.periodic;
  a.wall_w = a.wall_e = a.wall_n = 0;
  a.wall_s = d.wall_s;
  a.variant = 0;
  a.open = d.open;
  a.mixed = 0;
  a.t = 0.0;
  a.xmap0 = d.xmap0;
  a.ymap0 = d.ymap0;
  a.node_sides = 0;  // the item order already waits for the node pass
  a.mask = nullptr;
  a.box_x0 = a.box_x1 = a.box_y0 = a.box_y1 = 0;
  a.wall = P.wall;
  a.k = P.k;
  return a;
}

__device__ __forceinline__ NodeBcArgs persist_node_args(const PersistArgs& P, const PDomain& d,
                                                        int step, int st) {
  const int odd = (P.step0 + step) & 1;
  double* X = odd ? d.buf[1] : d.buf[0];
  double* Y = odd ? d.buf[0] : d.buf[1];
  NodeBcArgs a;
  a.utmp = X;
  a.u = st == 2 ? d.buf[2] : Y;
  a.f = d.f;
  a.dx = d.dx;
  a.dy = d.dy;
  a.rdx = d.rdx;
  a.rdy = d.rdy;
  a.t = 0.0;
  a.xmap0 = d.xmap0;
  a.ymap0 = d.ymap0;
  a.south_wall = d.south_wall;
  a.corners_y = d.corners_y;
  a.open_w = d.open_w;
  a.open_e = d.open_e;
  a.open_n = d.open_n;
  a.status = d.status;
  a.wall = P.wall;
  a.k = P.k;
  return a;
}

// wait until band b of domain d has completed `inst` stage-instances
__device__ __forceinline__ bool wait_band(const PersistArgs& P, const PDomain& d, int b,
                                          unsigned long long inst) {
  return wait_done(P, P.done + d.band0 + b, inst * (unsigned long long)P.sg[d.band0 + b]);
}

template <bool MIX>
__global__ void __launch_bounds__(32 * PW, 8) k_batch_persistent(const __grid_constant__ PersistArgs P) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned long long total = (unsigned long long)P.items_per_step * P.nsteps;
  for (;;) {
    unsigned long long it = 0;
    if (lane == 0) it = atomicAdd(P.next, 1ull);
    it = __shfl_sync(0xffffffffu, it, 0);
    if (it >= total || *(volatile unsigned int*)&P.ctl[0]) break;
    const int step = (int)(it / (unsigned long long)P.items_per_step);
    const PItem item = P.items[it % (unsigned long long)P.items_per_step];
    const PDomain& d = P.dom[item.dom];
    // stage-instances (3 per step) that precede this item's stage
    const unsigned long long inst = 3ull * (unsigned long long)step + (unsigned long long)(item.stage - 1);
    // Every lane checks the counters the item depends on: the counters read
    // together with relaxed loads and, if they are all ready (the usual
    // case), one acquire fence (the acquire pattern: strong reads, then
    // fence.acq_rel) -- one round trip; otherwise bounded waits, one counter
    // at a time.  (Lane 0 checking alone and the warp barrier passing the
    // order on measured 1.5x slower: divergent lanes wait on its branch.)
    // Strips that read no ghost cell of the node pass skip its wait
    // (`count` flags those that do).
    bool ok = true;
    if (item.type == PI_NODE) {
      for (int b = 0; b < d.nb && ok; b++) ok = wait_band(P, d, b, inst + 1);
    } else {
      const bool need_node = d.nn && (item.type != PI_STRIP || item.count);
      int bands[3];
      for (int o = -1; o <= 1; o++) {
        int bb = item.band + o;
        if (bb < 0 || bb >= d.nb) bb = d.periodic ? (bb + d.nb) % d.nb : item.band;
        bands[o + 1] = bb;
      }
      const unsigned long long c0 = load_relaxed(P.done + d.band0 + bands[0]);
      const unsigned long long c1 = load_relaxed(P.done + d.band0 + bands[1]);
      const unsigned long long c2 = load_relaxed(P.done + d.band0 + bands[2]);
      const unsigned long long cn = need_node ? load_relaxed(P.ndone + item.dom) : 0ull;
      const bool ready = c0 >= inst * (unsigned long long)P.sg[d.band0 + bands[0]] &&
                         c1 >= inst * (unsigned long long)P.sg[d.band0 + bands[1]] &&
                         c2 >= inst * (unsigned long long)P.sg[d.band0 + bands[2]] &&
                         cn >= (need_node ? inst * (unsigned long long)d.nn : 0ull);
      if (ready) {
        fence_acquire();
      } else {
        for (int o = 0; o < 3 && ok; o++) ok = wait_band(P, d, bands[o], inst);
        if (ok && need_node)
          ok = wait_done(P, P.ndone + item.dom, inst * (unsigned long long)d.nn);
      }
    }
    // a wait that ran out stops the warp (the launch is aborted)
    if (!__all_sync(0xffffffffu, ok)) break;
    if (item.type == PI_STRIP) {
      const StageArgs a = persist_stage_args(P, d, step, item.stage);
      const int c0 = BC + (item.index % d.sx) * SW;
      const int y0 = BC + item.band * P.h_rows;
      // the last band runs to the last interior row (it absorbs a remainder
      // of fewer than 2 rows, so that the rows a periodic field images into
      // the opposite ghost rows never span two bands)
      const int y1 = item.band == d.nb - 1 ? d.f.ny - BC : y0 + P.h_rows;
      strip_warp<1, true, MIX>(a, c0, y0, y1, warp);
    } else if (item.type == PI_GHOST) {
      if (lane < item.count)
        open_ghost_cell(persist_stage_args(P, d, step, item.stage), item.index + lane, 1);
    } else {
      node_bc_cell(persist_node_args(P, d, step, item.stage), item.index * 32 + lane);
    }
    // release: the warp barrier orders every lane's stores before lane 0,
    // whose fence (cumulative) precedes the counter increment.  The
    // counter's address is looked up again from the item table rather than
    // kept live across the work.
    __syncwarp();
    if (lane == 0 && (long long)it != P.withhold) {
      __threadfence();
      const PItem& done_item = P.items[it % (unsigned long long)P.items_per_step];
      atomicAdd(done_item.type == PI_NODE
                    ? P.ndone + done_item.dom
                    : P.done + P.dom[done_item.dom].band0 + done_item.band,
                1ull);
    }
  }
}

#undef ST
#undef UV
#undef NQ_
#undef FQ
#undef KQ

// launch; with `after_node_pass`, as a programmatic dependent of the node
// pass launched just before on `s` (it may start while the pass runs)
inline cudaError_t launch_after_node_pass(const void* fn, unsigned blocks, unsigned threads,
                                          size_t smem, cudaStream_t s, bool after_node_pass,
                                          void** args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = after_node_pass ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

template <int H, int WPC, int MINB, int MODE, bool MIX>
const void* strip_fn(int kind) {
  if (kind == K_WALL) return (const void*)k_strip<H, WPC, MINB, MODE, K_WALL, MIX>;
  if (kind == K_OPEN) return (const void*)k_strip<H, WPC, MINB, MODE, K_OPEN, MIX>;
  if (kind == K_WALL_OPEN) return (const void*)k_strip<H, WPC, MINB, MODE, K_WALL_OPEN, MIX>;
  return (const void*)k_strip<H, WPC, MINB, MODE, K_PLAIN, MIX>;
}

template <int H, int WPC, int MINB>
cudaError_t launch_strip_shape(const StageArgs& a, int mode, cudaStream_t s) {
  const size_t smem =
      (size_t)WPC * (a.mixed ? WARP_DOUBLES_MIX : WARP_DOUBLES) * sizeof(double);
  const bool wall = a.wall_w || a.wall_e || a.wall_s || a.wall_n;
  const int kind = a.open ? (wall ? K_WALL_OPEN : K_OPEN) : (wall ? K_WALL : K_PLAIN);
  const void* fn = a.mixed ? (mode == 0 ? strip_fn<H, WPC, MINB, 0, true>(kind)
                                        : strip_fn<H, WPC, MINB, 1, true>(kind))
                           : (mode == 0 ? strip_fn<H, WPC, MINB, 0, false>(kind)
                                        : strip_fn<H, WPC, MINB, 1, false>(kind));
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int sx = (a.f.nx - 2 * BC + SW - 1) / SW;
  const int sy = (a.f.ny - 2 * BC + H * WPC - 1) / (H * WPC);
  int ghost_ctas = a.open ? (open_ghost_count(a.f, a.open) + 32 * WPC - 1) / (32 * WPC) : 0;
  const unsigned blocks = (unsigned)ghost_ctas + (unsigned)sx * (unsigned)sy;
  StageArgs aa = a;
  void* args[] = {&aa, &ghost_ctas, &sx};
  return launch_after_node_pass(fn, blocks, 32 * WPC, smem, s, a.node_sides != 0, args);
}

template <int H, int WPC, int MINB, bool MIX>
const void* strip_batch_fn(int kind) {
  return kind == BK_WALL   ? (const void*)k_strip_batch<H, WPC, MINB, K_WALL_OPEN, MIX>
         : kind == BK_OPEN ? (const void*)k_strip_batch<H, WPC, MINB, K_OPEN, MIX>
                           : (const void*)k_strip_batch<H, WPC, MINB, K_PLAIN, MIX>;
}

template <int H, int WPC, int MINB>
cudaError_t launch_strip_batch_shape(BatchStageArgs& P, int kind, bool mixed, cudaStream_t s) {
  const size_t smem = (size_t)WPC * (mixed ? WARP_DOUBLES_MIX : WARP_DOUBLES) * sizeof(double);
  const void* fn = mixed ? strip_batch_fn<H, WPC, MINB, true>(kind)
                         : strip_batch_fn<H, WPC, MINB, false>(kind);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  long long ghost = 0, strips = 0;
  for (int i = 0; i < P.ndom; i++) {
    BatchDomain& d = P.d[i];
    d.sx = (d.f.nx - 2 * BC + SW - 1) / SW;
    const int sy = (d.f.ny - 2 * BC + H * WPC - 1) / (H * WPC);
    d.ghost0 = (int)ghost;
    d.strip0 = (int)strips;
    if (kind == BK_OPEN || kind == BK_WALL)
      ghost += (open_ghost_count(d.f, d.open) + 32 * WPC - 1) / (32 * WPC);
    strips += (long long)d.sx * sy;
  }
  if (ghost + strips > 0x7fffffffLL) return cudaErrorInvalidValue;
  P.ghost_ctas = (int)ghost;
  bool pdl = false;
  for (int i = 0; i < P.ndom; i++) pdl = pdl || P.d[i].node_sides != 0;
  void* args[] = {&P};
  return launch_after_node_pass(fn, (unsigned)(ghost + strips), 32 * WPC, smem, s, pdl, args);
}

}  // namespace

cudaError_t launch_batch_persistent(const PersistArgs& P, bool mixed, cudaStream_t s, int* ctas) {
  const size_t smem = (size_t)PW * (mixed ? WARP_DOUBLES_MIX : WARP_DOUBLES) * sizeof(double);
  const void* fn = mixed ? (const void*)k_batch_persistent<true> : (const void*)k_batch_persistent<false>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0, per_sm = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * PW, smem);
  if (e != cudaSuccess) return e;
  const int n = sms * (per_sm > 0 ? per_sm : 1);
  if (ctas) *ctas = n;
  PersistArgs pa = P;
  void* args[] = {&pa};
  return cudaLaunchKernel(fn, dim3((unsigned)n), dim3(32 * PW), args, smem, s);
}

cudaError_t launch_strip_batch(BatchStageArgs& P, int kind, int shape, bool mixed,
                               cudaStream_t s) {
  if (P.ndom <= 0) return cudaSuccess;
  if (P.ndom > BATCH_MAX) return cudaErrorInvalidValue;
  switch (shape) {
    case 0: return launch_strip_batch_shape<8, 4, 4>(P, kind, mixed, s);
    case 1: return launch_strip_batch_shape<16, 4, 4>(P, kind, mixed, s);
    case 2: return launch_strip_batch_shape<16, 4, 5>(P, kind, mixed, s);
    case 3: return launch_strip_batch_shape<16, 2, 8>(P, kind, mixed, s);
    case 4: return launch_strip_batch_shape<16, 8, 2>(P, kind, mixed, s);
  }
  return cudaErrorInvalidValue;
}

template <int H, int WPC, int MINB>
cudaError_t launch_strip_masked_shape(const StageArgs& a, cudaStream_t s) {
  const size_t smem = (size_t)WPC * WARP_DOUBLES * sizeof(double);
  const void* fn = (const void*)k_strip<H, WPC, MINB, 2, K_PLAIN, false>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int sx = (a.box_x1 - (a.box_x0 & ~1) + SW) / SW;
  const int sy = (a.box_y1 - a.box_y0 + H * WPC) / (H * WPC);
  int ghost_ctas = 0;
  StageArgs aa = a;
  void* args[] = {&aa, &ghost_ctas, &sx};
  return launch_after_node_pass(fn, (unsigned)sx * (unsigned)sy, 32 * WPC, smem, s, false, args);
}

// L(u) of a buffer-layer grid at its interior_pt points (MODE 2) over the
// border box [box_x0, box_x1] x [box_y0, box_y1] (box_x0, box_y0 >= BC:
// every copied row and column lies inside the grid).  Strips of 16 rows (2
// warps per CTA, 8 CTAs per SM) where they fill the GPU's 148 x 16 warp
// slots, else of 8 rows (4 warps per CTA) for twice the warps: layers are
// often thin bands.  Needs strip_layout_ok(a).
cudaError_t launch_strip_masked(const StageArgs& a, cudaStream_t s) {
  const long long sx = (a.box_x1 - (a.box_x0 & ~1) + SW) / SW;
  const long long warps16 = sx * ((a.box_y1 - a.box_y0 + 16) / 16);
  if (warps16 >= 148LL * 16) return launch_strip_masked_shape<16, 2, 8>(a, s);
  return launch_strip_masked_shape<8, 4, 4>(a, s);
}

// shape id -> (rows per warp, warps per CTA, minimum resident CTAs per SM
// requested from the register allocator)
cudaError_t launch_strip_stage(const StageArgs& a, int mode, int shape, cudaStream_t s) {
  switch (shape) {
    case 0: return launch_strip_shape<8, 4, 4>(a, mode, s);
    case 1: return launch_strip_shape<16, 4, 4>(a, mode, s);
    case 2: return launch_strip_shape<16, 4, 5>(a, mode, s);
    case 3: return launch_strip_shape<16, 2, 8>(a, mode, s);
    case 4: return launch_strip_shape<16, 8, 2>(a, mode, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace dim2d
