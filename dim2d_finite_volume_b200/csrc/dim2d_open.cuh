// dim2d_open.cuh -- open (Hedstrom, non-reflecting) boundary on sm_100a.
//
// For a field whose eight boundary sections are all `hedstrom_choice` of
// type bc_timedev (library_config.py:155-168), the ghost layers are
// time-integrated like the interior (field_abstract_class.f:244-270
// widens x/y_borders), with a time derivative built per ghost cell by
// bc_operators_hedstrom_xy_class.f:182-496:
//   * N/S ghost rows: (Fx_i - Fx_{i+1})/dx with x-face fluxes evaluated by
//     the y one-sided operator sets (R1/R0 on N, L0/L1 on S;
//     bc_operators_openbc_normal_class.f:563-713), plus the characteristic
//     y-direction term; E/W ghost columns are the transposed case;
//   * corners: characteristic x term + characteristic y term;
//   * characteristic term (hedstrom_xy_module.f:445-558): eigen-quantities
//     of the node itself (obc_eigenqties_bc), amplitudes of outgoing waves
//     from one-sided normal gradients, incoming ones set to zero, mapped
//     back through the conservative <- primitive Jacobian
//     (ns_vdw2d_prim_module.f:249-893).
// The presets that mix open sections with a south wall (wall_S_open,
// half_wall_S_open, library_config.py:118-150) integrate only their open
// sections (StageArgs::open mask); where an open W/E edge meets the wall
// corner, the corner's wall flux closes the edge's first interior row.
// One thread per ghost cell; the state is read straight from global memory
// (the ghost ring is a few rows, L2-resident), the output is written with
// the same RK3 stage update as the interior kernel.  Included by
// dim2d_open.cu (stand-alone ghost kernel) and dim2d_strip.cu (ghost
// cells fused into the stage launch as its first CTAs).
#pragma once
#include "dim2d_kernels.cuh"

// Device loads go through the read-only (non-coherent) path, except in a
// translation unit that defines DIM2D_COHERENT_LOADS: the persistent kernel
// reads fields that other SMs rewrite during the same launch, so its loads
// must be coherent (ld.global.cg, ordered by the acquire of its waits).
#if defined(__CUDA_ARCH__) && defined(DIM2D_COHERENT_LOADS)
#define DIM2D_LDG(p) __ldcg(p)
#elif defined(__CUDA_ARCH__)
#define DIM2D_LDG(p) __ldg(p)
#elif defined(DIM2D_LDG_HOST)
#define DIM2D_LDG(p) DIM2D_LDG_HOST(p)  // host emulation with checked reads
#else
#define DIM2D_LDG(p) (*(p))
#endif

namespace dim2d {

namespace {

// tangential operator variant of a face in a ghost row/column
enum TMode : int { T_INT = 0, T_L0 = 1, T_R0 = 2 };

struct Node {
  double r, mn, mt, e;
};

// Accessor in a face frame: n = coordinate along the face normal,
// t = along the face.  For x-faces (n = x) m_n = rho u; for y-faces m_n = rho v.
struct Frame {
  const double* __restrict__ u;
  Field f;
  int bx, by;  // node b (high side of the face)
  bool ydir;   // normal along y
  __host__ __device__ __forceinline__ size_t idx(int n, int t) const {
    const int x = ydir ? bx + t : bx + n;
    const int y = ydir ? by + n : by + t;
    return (size_t)y * f.pitch + x;
  }
  __host__ __device__ __forceinline__ Node node(int n, int t) const {
    const size_t o = idx(n, t);
    Node q;
    q.r = DIM2D_LDG(u + o);
    const double mx = DIM2D_LDG(u + o + f.plane), my = DIM2D_LDG(u + o + 2 * f.plane);
    q.mn = ydir ? my : mx;
    q.mt = ydir ? mx : my;
    q.e = DIM2D_LDG(u + o + 3 * f.plane);
    return q;
  }
  __host__ __device__ __forceinline__ double rho(int n, int t) const { return DIM2D_LDG(u + idx(n, t)); }
};

struct NP {  // primitives of a node in the frame
  double un, ut, p, tcl, cp;
};
__host__ __device__ __forceinline__ NP nprim(const Node& q, const DimConst& k) {
  const NodePrim p = node_prim(q.r, q.mn, q.mt, q.e, k);  // u <-> n, v <-> t
  NP o;
  o.un = p.u;
  o.ut = p.v;
  o.p = p.p;
  o.tcl = p.tcl;
  o.cp = p.cp;
  return o;
}

// Tcap at frame node (n,t): centred normal gradient, tangential gradient
// per mode (sd_operators_fd_module.f:71-153, 182-450)
__host__ __device__ __forceinline__ double tcap_at(const Frame& F, int n, int t, int tm, double rdn,
                                          double rdt) {
  const double r = F.rho(n, t);
  const double gn = 0.5 * rdn * (F.rho(n + 1, t) - F.rho(n - 1, t));
  double gt;
  if (tm == T_INT) gt = 0.5 * rdt * (F.rho(n, t + 1) - F.rho(n, t - 1));
  else if (tm == T_R0) gt = rdt * (r - F.rho(n, t - 1));
  else gt = rdt * (F.rho(n, t + 1) - r);
  return 0.5 / r * (gn * gn + gt * gt);
}

// Face inputs at the face between frame nodes a = (-1, 0) and b = (0, 0)
// with the tangential operators of mode tm (the normal operators are the
// interior ones in every set used here: y_{L0,L1,R1,R0} change only
// y-derivatives of x-faces, x_{...} only x-derivatives of y-faces);
// *tcl_b = classical temperature_eff of node b.
__host__ __device__ void frame_face_in(const Frame& F, int tm, double rdn, double rdt,
                                       const DimConst& k, FaceIn& fi, double* tcl_b) {
  const Node a = F.node(-1, 0), b = F.node(0, 0);
  const NP pa = nprim(a, k), pb = nprim(b, k);
  *tcl_b = pb.tcl;
  fi.ra = a.r; fi.rb = b.r;
  fi.mna = a.mn; fi.mnb = b.mn;
  fi.mta = a.mt; fi.mtb = b.mt;
  fi.ea = a.e; fi.eb = b.e;
  fi.una = pa.un; fi.unb = pb.un;
  fi.uta = pa.ut; fi.utb = pb.ut;
  fi.pa = pa.p; fi.pb = pb.p;
  fi.ta = pa.tcl; fi.tb = pb.tcl;
  fi.ca = pa.cp; fi.cb = pb.cp;
  fi.ka = tcap_at(F, -1, 0, tm, rdn, rdt);
  fi.kb = tcap_at(F, 0, 0, tm, rdn, rdt);
  fi.drn = rdn * (b.r - a.r);
  fi.dunn = rdn * (pb.un - pa.un);
  fi.dutn = rdn * (pb.ut - pa.ut);
  fi.dtn = rdn * (pb.tcl - pa.tcl);
  fi.dkn = rdn * (fi.kb - fi.ka);
  const double d2n = 0.5 * rdn * rdn * (F.rho(-2, 0) - a.r - b.r + F.rho(1, 0));
  // tangential pairs (a,b) at rows t-2..t+2 as needed
  double drt, dunt, dutt, d2t;
  if (tm == T_INT) {
    const Node ap = F.node(-1, 1), bp = F.node(0, 1), am = F.node(-1, -1), bm = F.node(0, -1);
    const NP pap = nprim(ap, k), pbp = nprim(bp, k), pam = nprim(am, k), pbm = nprim(bm, k);
    const double q = 0.25 * rdt;
    drt = q * ((ap.r + bp.r) - (am.r + bm.r));
    dunt = q * ((pap.un + pbp.un) - (pam.un + pbm.un));
    dutt = q * ((pap.ut + pbp.ut) - (pam.ut + pbm.ut));
    d2t = 0.5 * rdt * rdt * ((am.r + bm.r) - 2.0 * (a.r + b.r) + (ap.r + bp.r));
  } else if (tm == T_R0) {  // sd_operators_y_oneside_R0_class.f:229-331 (and x mirror)
    const Node am = F.node(-1, -1), bm = F.node(0, -1);
    const NP pam = nprim(am, k), pbm = nprim(bm, k);
    const double h = 0.5 * rdt;
    drt = h * ((a.r + b.r) - (am.r + bm.r));
    dunt = h * ((pa.un + pb.un) - (pam.un + pbm.un));
    dutt = h * ((pa.ut + pb.ut) - (pam.ut + pbm.ut));
    d2t = 0.5 * rdt * rdt * ((F.rho(-1, -2) + F.rho(0, -2)) - 2.0 * (am.r + bm.r) + (a.r + b.r));
  } else {  // T_L0: sd_operators_y_oneside_L0_class.f:229-331 (and x mirror)
    const Node ap = F.node(-1, 1), bp = F.node(0, 1);
    const NP pap = nprim(ap, k), pbp = nprim(bp, k);
    const double h = 0.5 * rdt;
    drt = h * ((ap.r + bp.r) - (a.r + b.r));
    dunt = h * ((pap.un + pbp.un) - (pa.un + pb.un));
    dutt = h * ((pap.ut + pbp.ut) - (pa.ut + pb.ut));
    d2t = 0.5 * rdt * rdt * ((a.r + b.r) - 2.0 * (ap.r + bp.r) + (F.rho(-1, 2) + F.rho(0, 2)));
  }
  fi.drt = drt;
  fi.dunt = dunt;
  fi.dutt = dutt;
  fi.lap = d2n + d2t;
}

// Interior-formula flux at that face (flux_x/y_oneside with the set of tm)
__host__ __device__ void frame_face_flux(const Frame& F, int tm, double rdn, double rdt,
                                         const DimConst& k, double out[4]) {
  FaceIn fi;
  double tcl_b;
  frame_face_in(F, tm, rdn, rdt, k, fi, &tcl_b);
  face_flux(fi, k, out);
}

// Wall flux at a y-face on the south wall (node b = first interior row):
// the flux of the wall corner sections, bc_operators_wall_xy_class.f:
// 702-854 (SW: x_oneside_L0 set in column 1, L1 in column 2; SE: R1 in
// column nx-1, R0 in column nx) with compute_wall_flux_y,
// wall_xy_equilibrium_module.f:445-908.  Of the set's operators the wall
// flux uses the tangential density gradient and second derivative (mode
// tm) and the temperature of node b with the tangential gradient of mode
// tm (temperature_eff with gradient_x_x_oneside_L0/R0 in the outer column).
__host__ __device__ void frame_wall_flux_s(const Frame& F, int tm, double rdn, double rdt,
                                           double dn, double q, const DimConst& k,
                                           double out[4]) {
  FaceIn fi;
  double tcl_b;
  frame_face_in(F, tm, rdn, rdt, k, fi, &tcl_b);
  const double tl = k.c38cv * (tcl_b - k.iwe * fi.kb);
  wall_face_flux(fi, tl, dn, q, q, k, out);
}

// hedstrom_xy_module.f:445-558 with obc_eigenqties_bc.  q = conservative
// state of the node, g = one-sided normal gradients of (rho, u, v, P);
// ydir = normal along y; right = E or N side.  Output: conservative
// time derivative contribution.
__host__ __device__ void char_term(const double q[4], const double g[4], bool ydir, bool right,
                          const DimConst& k, double td[4]) {
  const double md = q[0];
  const double ux = q[1] / q[0], uy = q[2] / q[0];
  const double P = 3.0 / ((3.0 - md) * k.cv_r) * (q[3] - 0.5 * md * (ux * ux + uy * uy) +
                                                  3.0 * (md * md)) - 3.0 * (md * md);
  const double c = sound_speed(q[0], q[1], q[2], q[3], k);
  const double un = ydir ? uy : ux;
  const double ev[4] = {un, un, un - c, un + c};
  const double q_c = 0.5 * md * c;
  const double ic2 = 1.0 / (c * c);
  // left eigenvectors (columns), ns_vdw2d_prim_module.f:574-635 / 744-805
  double lg[4];
  if (!ydir) {
    lg[0] = g[2];
    lg[1] = g[0] - ic2 * g[3];
    lg[2] = -q_c * g[1] + 0.5 * g[3];
    lg[3] = q_c * g[1] + 0.5 * g[3];
  } else {
    lg[0] = g[1];
    lg[1] = g[0] - ic2 * g[3];
    lg[2] = -q_c * g[2] + 0.5 * g[3];
    lg[3] = q_c * g[2] + 0.5 * g[3];
  }
  double amp[4];
#pragma unroll
  for (int m = 0; m < 4; m++) {
    const bool incoming = right ? ev[m] <= 0.0 : ev[m] >= 0.0;  // openbc_operators_module.f:97-136
    amp[m] = incoming ? 0.0 : -ev[m] * lg[m];
  }
  // right eigenvectors (rows), ns_vdw2d_prim_module.f:657-722 / 827-893
  const double iqc = 1.0 / (md * c);
  double tp[4];
  tp[0] = amp[1] + ic2 * amp[2] + ic2 * amp[3];
  tp[3] = amp[2] + amp[3];
  if (!ydir) {
    tp[1] = -iqc * amp[2] + iqc * amp[3];
    tp[2] = amp[0];
  } else {
    tp[1] = amp[0];
    tp[2] = -iqc * amp[2] + iqc * amp[3];
  }
  // conservative <- primitive Jacobian, ns_vdw2d_prim_module.f:249-320
  const double dEdrho = 0.5 * (ux * ux + uy * uy) - 6.0 * md -
                        1.0 / 3.0 * k.cv_r * (P + 9.0 * (md - 2.0) * md);
  td[0] = tp[0];
  td[1] = tp[0] * ux + tp[1] * md;
  td[2] = tp[0] * uy + tp[2] * md;
  td[3] = tp[0] * dEdrho + tp[1] * (md * ux) + tp[2] * (md * uy) + tp[3] * (k.cv_r * (1.0 - md / 3.0));
}

__host__ __device__ __forceinline__ void load4(const double* u, const Field& f, int x, int y, double q[4]) {
  const size_t o = (size_t)y * f.pitch + x;
  q[0] = DIM2D_LDG(u + o);
  q[1] = DIM2D_LDG(u + o + f.plane);
  q[2] = DIM2D_LDG(u + o + 2 * f.plane);
  q[3] = DIM2D_LDG(u + o + 3 * f.plane);
}

// one-sided normal gradient of (rho, u, v, P) at node (x,y):
// R0 = (phi(n) - phi(n-1))/dn, L0 = (phi(n+1) - phi(n))/dn
__host__ __device__ void prim_gradient(const double* u, const Field& f, int x, int y, bool ydir, bool right,
                              double rdn, const DimConst& k, double g[4]) {
  const int sx = ydir ? 0 : 1, sy = ydir ? 1 : 0;
  double q0[4], q1[4];
  if (right) {
    load4(u, f, x - sx, y - sy, q0);
    load4(u, f, x, y, q1);
  } else {
    load4(u, f, x, y, q0);
    load4(u, f, x + sx, y + sy, q1);
  }
  const NodePrim p0 = node_prim(q0[0], q0[1], q0[2], q0[3], k);
  const NodePrim p1 = node_prim(q1[0], q1[1], q1[2], q1[3], k);
  g[0] = rdn * (q1[0] - q0[0]);
  g[1] = rdn * (p1.u - p0.u);
  g[2] = rdn * (p1.v - p0.v);
  g[3] = rdn * (p1.p - p0.p);
}

}  // namespace

// cells of ghost section s (0..3 = S, N, W, E edges, 4..7 = SW, SE, NW,
// NE corners; bit s of an OPEN_* mask)
inline __host__ __device__ int open_section_cells(const Field& f, int s) {
  if (s < 2) return BC * (f.nx - 2 * BC);
  if (s < 4) return BC * (f.ny - 2 * BC);
  return BC * BC;
}

// number of ghost cells of the sections in `mask`
inline __host__ __device__ int open_ghost_count(const Field& f, int mask) {
  int n = 0;
  for (int s = 0; s < 8; s++)
    if (mask >> s & 1) n += open_section_cells(f, s);
  return n;
}

// Ghost cell number m of the open sections a.open: time derivative
// (mode 0) or RK stage update (mode 1) written to a.uout.  Cells are
// numbered section by section in the order S edge, N edge (BC rows of ex
// cells each), W edge, E edge (BC columns of ey cells each), SW, SE, NW,
// NE corners (BC x BC), skipping sections outside the mask.  With a wall on
// the south side (a.wall_s; its corner sections are wall sections), the
// bottom y-face of the first interior row of an open W or E edge carries
// the wall corner flux instead of the open-edge flux: the open edge's own
// flux range starts one face higher (check_y_flux_interactions,
// bc_operators_openbc_class.f:437-551) and the wall corner operator
// supplies that face.
inline __host__ __device__ void open_ghost_cell(const StageArgs& a, int m, int mode) {
  const Field f = a.f;
  const int ex = f.nx - 2 * BC, ey = f.ny - 2 * BC;  // interior extents
  const int mask = a.open;
  if (m < 0) return;
  int sec = 0;
  for (; sec < 8; sec++) {
    if (!(mask >> sec & 1)) continue;
    const int c = open_section_cells(f, sec);
    if (m < c) break;
    m -= c;
  }
  if (sec == 8) return;
  const DimConst& k = a.k;
  int x, y;
  double L[4];
  double q[4];
  if (sec < 2) {  // N or S edge cell: x-faces in the ghost row
    const bool north = sec == 1;
    const int r = m;
    x = BC + r % ex;
    const int row = r / ex;  // 0 or 1
    y = north ? f.ny - BC + row : row;
    // operator set of this ghost row: N: R1 (row ny-2) = interior, R0 (row ny-1);
    // S: L0 (row 0), L1 (row 1) = interior
    int tm = T_INT;
    if (north && y == f.ny - 1) tm = T_R0;
    if (!north && y == 0) tm = T_L0;
    double Fl[4], Fr[4];
    Frame Fa{a.uin, f, x, y, false};
    frame_face_flux(Fa, tm, a.rdx, a.rdy, k, Fl);
    Frame Fb{a.uin, f, x + 1, y, false};
    frame_face_flux(Fb, tm, a.rdx, a.rdy, k, Fr);
    double g[4], ch[4];
    prim_gradient(a.uin, f, x, y, true, north, a.rdy, k, g);
    load4(a.uin, f, x, y, q);
    char_term(q, g, true, north, k, ch);
    // hedstrom_xy_module.f:290-303
#pragma unroll
    for (int v = 0; v < 4; v++) L[v] = (Fl[v] - Fr[v]) * a.rdx + ch[v];
  } else if (sec < 4) {  // E or W edge cell: y-faces in the ghost column
    const bool east = sec == 3;
    const int r = m;
    y = BC + r % ey;
    const int col = r / ey;
    x = east ? f.nx - BC + col : col;
    int tm = T_INT;
    if (east && x == f.nx - 1) tm = T_R0;
    if (!east && x == 0) tm = T_L0;
    double Gb[4], Gt[4];
    Frame Fa{a.uin, f, x, y, true};
    if (a.wall_s && y == BC)
      frame_wall_flux_s(Fa, tm, a.rdy, a.rdx, a.dy, wall_heat_flux(a.wall, a.xmap0 + x * a.dx),
                        k, Gb);
    else
      frame_face_flux(Fa, tm, a.rdy, a.rdx, k, Gb);
    Frame Fb{a.uin, f, x, y + 1, true};
    frame_face_flux(Fb, tm, a.rdy, a.rdx, k, Gt);
    double g[4], ch[4];
    prim_gradient(a.uin, f, x, y, false, east, a.rdx, k, g);
    load4(a.uin, f, x, y, q);
    char_term(q, g, false, east, k, ch);
    // hedstrom_xy_module.f:204-216; y-face frame order is (mass, m_y, m_x, E)
    L[0] = ch[0] + (Gb[0] - Gt[0]) * a.rdy;
    L[1] = ch[1] + (Gb[2] - Gt[2]) * a.rdy;
    L[2] = ch[2] + (Gb[1] - Gt[1]) * a.rdy;
    L[3] = ch[3] + (Gb[3] - Gt[3]) * a.rdy;
  } else {  // corner cell: characteristic x + characteristic y
    const int c = sec - 4, r = m;
    const bool east = c & 1, north = c >> 1;
    x = (east ? f.nx - BC : 0) + r % BC;
    y = (north ? f.ny - BC : 0) + r / BC;
    double gx[4], gy[4], cx[4], cy[4];
    prim_gradient(a.uin, f, x, y, false, east, a.rdx, k, gx);
    prim_gradient(a.uin, f, x, y, true, north, a.rdy, k, gy);
    load4(a.uin, f, x, y, q);
    char_term(q, gx, false, east, k, cx);
    char_term(q, gy, true, north, k, cy);
#pragma unroll
    for (int v = 0; v < 4; v++) L[v] = cx[v] + cy[v];
  }
  if (k.gravity_ac) {  // openbc_operators_module.f:354-372
    L[2] += -q[0] * k.gravity;
    L[3] += -q[2] * k.gravity;
  }
  const size_t o = (size_t)y * f.pitch + x;
#pragma unroll
  for (int v = 0; v < 4; v++) {
    double out;
    if (mode == 0) out = L[v];
    else if (a.stage == 1) out = q[v] + a.dt * L[v];
    else out = a.b * DIM2D_LDG(a.u0 + o + v * f.plane) + (1.0 - a.b) * (q[v] + a.dt * L[v]);
    a.uout[o + v * f.plane] = out;
  }
}

}  // namespace dim2d
