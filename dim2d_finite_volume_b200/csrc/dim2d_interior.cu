// dim2d_interior.cu -- fused interior RK3 stage for sm_100a.
//
// One CTA owns a TILE_X x TILE_Y block of interior cells and performs, in
// shared memory, the whole chain that the reference spreads over
// compute_time_dev and compute_Nth_step:
//   1. stage the (TX+4) x (TY+4) x 4 halo tile of the input state
//      (stencil half-width 2, sd_operators_class.f get_bc_size = 2);
//   2. per-node primitives on the (TX+2) x (TY+2) ring the faces touch
//      (velocity, classical pressure/temperature, 1/(3-rho), Tcap);
//   3. the x-face fluxes (TX+1) x TY and y-face fluxes TX x (TY+1)
//      (pmodel_eq_class.f:1073-1180, dim2d_fluxes_module.f);
//   4. the flux divergence plus body force (td_operators_class.f:181-194)
//      and the stage update (rk3tvd_steps_module.f:52-100, 205-269,
//      424-490), written straight to the output copy of the field.
// Periodic domains also write the ghost images of the edge cells
// (periodic_xy/bc_operators_class.f:156-199), so a periodic stage is one
// launch with no separate boundary pass.
//
// HBM traffic per stage: read the input state once (+halo re-reads that
// hit L2), read u^n once for stages 2-3, write the output once.
#include "dim2d_kernels.cuh"

namespace dim2d {

namespace {

constexpr int TX = TILE_X, TY = TILE_Y;
constexpr int LX = TX + 4, LY = TY + 4;  // halo tile
constexpr int PX = TX + 2, PY = TY + 2;  // primitive ring
constexpr int NT = TX * TY;
constexpr int NFX = (TX + 1) * TY;
constexpr int NFY = TX * (TY + 1);
constexpr int SM_RAW = 4 * LX * LY;
constexpr int SM_PRIM = 6 * PX * PY;
constexpr int SM_FX = 4 * TY * (TX + 1);
constexpr int SM_FY = 4 * (TY + 1) * TX;
constexpr int SM_DOUBLES = SM_RAW + SM_PRIM + SM_FX + SM_FY;

// mode: 0 = write L(u) (time derivative), 1 = RK stage update,
// 2 = L(u) of a buffer-layer grid: tiles over [box_x0, box_x1] x
// [box_y0, box_y1], written where the grdpts_id map is interior_pt.  A face
// whose stencil reaches a no_pt node (whatever it holds) feeds only points
// that are not interior_pt: every point within two of an interior_pt point is
// a boundary point of the layer.
// Four 256-thread CTAs per SM (64 registers, no spills; 4 x 47.8 KB of shared
// memory): with three, the face pass left the FP64 pipe waiting on latency.
template <int MODE, bool WALL>
__global__ void __launch_bounds__(NT, 4) k_interior(StageArgs a) {
  extern __shared__ __align__(16) double sm[];
  double* sR = sm;
  double* sMx = sR + LX * LY;
  double* sMy = sMx + LX * LY;
  double* sE = sMy + LX * LY;
  double* sU = sE + LX * LY;
  double* sV = sU + PX * PY;
  double* sP = sV + PX * PY;
  double* sT = sP + PX * PY;
  double* sC = sT + PX * PY;
  double* sK = sC + PX * PY;
  double* sFx = sK + PX * PY;
  double* sFy = sFx + SM_FX;

  const Field f = a.f;
  const int x0 = (MODE == 2 ? a.box_x0 : BC) + blockIdx.x * TX;
  const int y0 = (MODE == 2 ? a.box_y0 : BC) + blockIdx.y * TY;
  const int tid = threadIdx.x;

  // 1. halo tile of the input state (rows are contiguous in HBM)
  for (int m = tid; m < LX * LY; m += NT) {
    const int lx = m % LX, ly = m / LX;
    const int gx = x0 - 2 + lx, gy = y0 - 2 + ly;
    double r = 1.0, mx = 0.0, my = 0.0, e = 0.0;  // benign values past the field edge
    if (gx < f.nx && gy < f.ny) {
      const size_t o = (size_t)gy * f.pitch + gx;
      r = __ldg(a.uin + o);
      mx = __ldg(a.uin + o + f.plane);
      my = __ldg(a.uin + o + 2 * f.plane);
      e = __ldg(a.uin + o + 3 * f.plane);
    }
    sR[m] = r;
    sMx[m] = mx;
    sMy[m] = my;
    sE[m] = e;
  }
  __syncthreads();

  // 2. primitives on the ring
  const DimConst& k = a.k;
  const double hrdx = 0.5 * a.rdx, hrdy = 0.5 * a.rdy;
  for (int m = tid; m < PX * PY; m += NT) {
    const int px = m % PX, py = m / PX;
    const int o = (py + 1) * LX + (px + 1);
    const NodePrim q = node_prim(sR[o], sMx[o], sMy[o], sE[o], k);
    sU[m] = q.u;
    sV[m] = q.v;
    sP[m] = q.p;
    sT[m] = q.tcl;
    sC[m] = q.cp;
    sK[m] = node_tcap(sR[o], sR[o - 1], sR[o + 1], sR[o - LX], sR[o + LX], hrdx, hrdy);
  }
  __syncthreads();

  // 3. face fluxes
  const double rdx = a.rdx, rdy = a.rdy;
  const double q_rdx = 0.25 * rdx, q_rdy = 0.25 * rdy;
  const double h_rdx2 = 0.5 * rdx * rdx, h_rdy2 = 0.5 * rdy * rdy;
  for (int m = tid; m < NFX + NFY; m += NT) {
    FaceIn fi;
    double F[4];
    if (m < NFX) {
      // x-face between nodes L=(fx-1,fy) and R=(fx,fy) of the tile
      const int fx = m % (TX + 1), fy = m / (TX + 1);
      const int pL = (fy + 1) * PX + fx, pR = pL + 1;
      const int oL = (fy + 2) * LX + fx + 1, oR = oL + 1;
      fi.ra = sR[oL]; fi.rb = sR[oR];
      fi.mna = sMx[oL]; fi.mnb = sMx[oR];
      fi.mta = sMy[oL]; fi.mtb = sMy[oR];
      fi.ea = sE[oL]; fi.eb = sE[oR];
      fi.una = sU[pL]; fi.unb = sU[pR];
      fi.uta = sV[pL]; fi.utb = sV[pR];
      fi.pa = sP[pL]; fi.pb = sP[pR];
      fi.ta = sT[pL]; fi.tb = sT[pR];
      fi.ca = sC[pL]; fi.cb = sC[pR];
      fi.ka = sK[pL]; fi.kb = sK[pR];
      fi.drn = rdx * (fi.rb - fi.ra);
      fi.drt = q_rdy * ((sR[oL + LX] + sR[oR + LX]) - (sR[oL - LX] + sR[oR - LX]));
      fi.dunn = rdx * (fi.unb - fi.una);
      fi.dunt = q_rdy * ((sU[pL + PX] + sU[pR + PX]) - (sU[pL - PX] + sU[pR - PX]));
      fi.dutn = rdx * (fi.utb - fi.uta);
      fi.dutt = q_rdy * ((sV[pL + PX] + sV[pR + PX]) - (sV[pL - PX] + sV[pR - PX]));
      const double d2n = h_rdx2 * (sR[oL - 1] - sR[oL] - sR[oR] + sR[oR + 1]);
      const double d2t = h_rdy2 * ((sR[oL - LX] + sR[oR - LX]) - 2.0 * (sR[oL] + sR[oR]) +
                                   (sR[oL + LX] + sR[oR + LX]));
      fi.lap = d2n + d2t;
      fi.dtn = rdx * (fi.tb - fi.ta);
      fi.dkn = rdx * (fi.kb - fi.ka);
      const int gxf = x0 + fx;  // face between columns gxf-1 and gxf
      const bool w_face = WALL && a.wall_w && gxf == BC;
      const bool e_face = WALL && a.wall_e && gxf == f.nx - BC;
      if (w_face || e_face) {
        // bc_operators_wall_xy_class.f:751-771: wall x-face; the low
        // temperature is taken on the interior side (:473-490)
        const int p = w_face ? pR : pL;
        const double tl = k.c38cv * (sT[p] - k.iwe * sK[p]);
        const double q = wall_heat_flux(a.wall, a.xmap0 + gxf * a.dx);
        wall_face_flux(fi, tl, a.dx, q, w_face ? q : -q, k, F);
      } else {
        face_flux(fi, k, F);
      }
      const int o = fy * (TX + 1) + fx;
      sFx[o] = F[0];
      sFx[o + TY * (TX + 1)] = F[1];
      sFx[o + 2 * TY * (TX + 1)] = F[2];
      sFx[o + 3 * TY * (TX + 1)] = F[3];
    } else {
      // y-face between nodes B=(gx,gy-1) and T=(gx,gy) of the tile
      const int mm = m - NFX;
      const int gx = mm % TX, gy = mm / TX;
      const int pB = gy * PX + gx + 1, pT = pB + PX;
      const int oB = (gy + 1) * LX + gx + 2, oT = oB + LX;
      fi.ra = sR[oB]; fi.rb = sR[oT];
      fi.mna = sMy[oB]; fi.mnb = sMy[oT];
      fi.mta = sMx[oB]; fi.mtb = sMx[oT];
      fi.ea = sE[oB]; fi.eb = sE[oT];
      fi.una = sV[pB]; fi.unb = sV[pT];
      fi.uta = sU[pB]; fi.utb = sU[pT];
      fi.pa = sP[pB]; fi.pb = sP[pT];
      fi.ta = sT[pB]; fi.tb = sT[pT];
      fi.ca = sC[pB]; fi.cb = sC[pT];
      fi.ka = sK[pB]; fi.kb = sK[pT];
      fi.drn = rdy * (fi.rb - fi.ra);
      fi.drt = q_rdx * ((sR[oB + 1] + sR[oT + 1]) - (sR[oB - 1] + sR[oT - 1]));
      fi.dunn = rdy * (fi.unb - fi.una);
      fi.dunt = q_rdx * ((sV[pB + 1] + sV[pT + 1]) - (sV[pB - 1] + sV[pT - 1]));
      fi.dutn = rdy * (fi.utb - fi.uta);
      fi.dutt = q_rdx * ((sU[pB + 1] + sU[pT + 1]) - (sU[pB - 1] + sU[pT - 1]));
      const double d2n = h_rdy2 * (sR[oB - LX] - sR[oB] - sR[oT] + sR[oT + LX]);
      const double d2t = h_rdx2 * ((sR[oB - 1] + sR[oT - 1]) - 2.0 * (sR[oB] + sR[oT]) +
                                   (sR[oB + 1] + sR[oT + 1]));
      fi.lap = d2n + d2t;
      fi.dtn = rdy * (fi.tb - fi.ta);
      fi.dkn = rdy * (fi.kb - fi.ka);
      const int gyf = y0 + gy;  // face between rows gyf-1 and gyf
      const bool s_face = WALL && a.wall_s && gyf == BC;
      const bool n_face = WALL && a.wall_n && gyf == f.ny - BC;
      if (s_face || n_face) {
        // bc_operators_wall_xy_class.f:729-749: wall y-face (:818-852)
        const int p = s_face ? pT : pB;
        const double tl = k.c38cv * (sT[p] - k.iwe * sK[p]);
        const double q = wall_heat_flux(a.wall, a.xmap0 + (x0 + gx) * a.dx);
        wall_face_flux(fi, tl, a.dy, q, s_face ? q : -q, k, F);
      } else {
        face_flux(fi, k, F);
      }
      const int o = gy * TX + gx;
      sFy[o] = F[0];
      sFy[o + (TY + 1) * TX] = F[2];      // momentum_x is tangential on a y-face
      sFy[o + 2 * (TY + 1) * TX] = F[1];  // momentum_y is normal
      sFy[o + 3 * (TY + 1) * TX] = F[3];
    }
  }
  __syncthreads();

  // 4. divergence + body force + stage update
  const int tx = tid % TX, ty = tid / TX;
  const int gx = x0 + tx, gy = y0 + ty;
  if (gx > f.nx - 1 - BC || gy > f.ny - 1 - BC) return;
  const int o = (ty + 2) * LX + tx + 2;
  const double uc[4] = {sR[o], sMx[o], sMy[o], sE[o]};
  const size_t go = (size_t)gy * f.pitch + gx;
  if (MODE == 2 && (gx > a.box_x1 || gy > a.box_y1 || __ldg(a.mask + go) != 1)) return;
  // periodic images of this cell in the ghost layers
  int ix2 = -1, iy2 = -1;
  if (a.periodic) {
    const int px = f.nx - 2 * BC, py = f.ny - 2 * BC;
    if (gx < 2 * BC) ix2 = gx + px;
    else if (gx >= f.nx - 2 * BC) ix2 = gx - px;
    if (gy < 2 * BC) iy2 = gy + py;
    else if (gy >= f.ny - 2 * BC) iy2 = gy - py;
  }
#pragma unroll
  for (int v = 0; v < 4; v++) {
    double L = (sFx[v * TY * (TX + 1) + ty * (TX + 1) + tx] -
                sFx[v * TY * (TX + 1) + ty * (TX + 1) + tx + 1]) * rdx +
               (sFy[v * (TY + 1) * TX + ty * TX + tx] -
                sFy[v * (TY + 1) * TX + (ty + 1) * TX + tx]) * rdy;
    if (k.gravity_ac) {  // pmodel_eq_class.f:1889-1904
      if (v == 2) L += -uc[0] * k.gravity;
      if (v == 3) L += -uc[2] * k.gravity;
    }
    double out;
    if (MODE != 1) {
      out = L;
    } else if (a.stage == 1) {
      out = uc[v] + a.dt * L;
    } else {
      const double u0 = __ldg(a.u0 + go + v * f.plane);
      out = a.b * u0 + (1.0 - a.b) * (uc[v] + a.dt * L);
    }
    double* dst = a.uout + v * f.plane;
    dst[go] = out;
    if (MODE == 1 && a.periodic) {
      if (ix2 >= 0) dst[(size_t)gy * f.pitch + ix2] = out;
      if (iy2 >= 0) {
        dst[(size_t)iy2 * f.pitch + gx] = out;
        if (ix2 >= 0) dst[(size_t)iy2 * f.pitch + ix2] = out;
      }
    }
  }
}

// Periodic ghost fill, equivalent to the reference's x pass over the
// interior rows followed by the y pass over all columns
// (periodic_xy/bc_operators_class.f:177-208).
__global__ void k_periodic_ghosts(double* u, Field f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= f.nx || j >= f.ny) return;
  const bool gx = i < BC || i >= f.nx - BC;
  const bool gy = j < BC || j >= f.ny - BC;
  if (!gx && !gy) return;
  const int px = f.nx - 2 * BC, py = f.ny - 2 * BC;
  int si = i, sj = j;
  if (i < BC) si = i + px;
  else if (i >= f.nx - BC) si = i - px;
  if (j < BC) sj = j + py;
  else if (j >= f.ny - BC) sj = j - py;
  for (int v = 0; v < 4; v++)
    u[v * f.plane + (size_t)j * f.pitch + i] = u[v * f.plane + (size_t)sj * f.pitch + si];
}

__global__ void k_fill(double* p, double v, size_t n) {
  for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < n;
       m += (size_t)gridDim.x * blockDim.x)
    p[m] = v;
}

// max over interior nodes of c + |u| (dim2d_prim_module.f:1179-1215):
// warp-shuffle reduction, one atomic per warp on the IEEE bit pattern
// (non-negative doubles order like their unsigned integer bits).
__global__ void k_cfl_max(const double* __restrict__ u, Field f, DimConst k,
                          unsigned long long* out) {
  const int ni = f.nx - 2 * BC, nj = f.ny - 2 * BC;
  double best = 0.0;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < ni * nj; m += gridDim.x * blockDim.x) {
    const int i = BC + m % ni, j = BC + m / ni;
    const size_t o = (size_t)j * f.pitch + i;
    const double r = u[o], mx = u[o + f.plane], my = u[o + 2 * f.plane], e = u[o + 3 * f.plane];
    const double c = sound_speed(r, mx, my, e, k);
    const double s = c + sqrt((mx / r) * (mx / r) + (my / r) * (my / r));
    best = fmax(best, s);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, off));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

}  // namespace

size_t interior_smem_bytes() { return SM_DOUBLES * sizeof(double); }

// The dynamic shared-memory opt-in is a per-device function attribute.
static cudaError_t set_smem_attr() {
  static bool done[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  const int bytes = (int)interior_smem_bytes();
  const void* fns[5] = {(const void*)k_interior<0, false>, (const void*)k_interior<1, false>,
                        (const void*)k_interior<0, true>, (const void*)k_interior<1, true>,
                        (const void*)k_interior<2, false>};
  for (const void* fn : fns) {
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    // four resident CTAs need the largest shared-memory carveout
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
  }
  if (dev >= 0 && dev < 64) done[dev] = true;
  return cudaSuccess;
}

template <int MODE>
static cudaError_t launch_mode(const StageArgs& a, cudaStream_t s) {
  if (stage_uses_strip(a)) return launch_strip_stage(a, MODE, strip_shape_of(a), s);
  cudaError_t e = set_smem_attr();
  if (e != cudaSuccess) return e;
  dim3 grid((a.f.nx - 2 * BC + TX - 1) / TX, (a.f.ny - 2 * BC + TY - 1) / TY);
  if (a.wall_w || a.wall_e || a.wall_s || a.wall_n)
    k_interior<MODE, true><<<grid, NT, interior_smem_bytes(), s>>>(a);
  else
    k_interior<MODE, false><<<grid, NT, interior_smem_bytes(), s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_interior_stage(const StageArgs& a, cudaStream_t s) {
  return launch_mode<1>(a, s);
}

cudaError_t launch_time_dev(const StageArgs& a, cudaStream_t s) { return launch_mode<0>(a, s); }

cudaError_t launch_time_dev_masked(const StageArgs& a, cudaStream_t s) {
  if (strip_layout_ok(a)) return launch_strip_masked(a, s);
  cudaError_t e = set_smem_attr();
  if (e != cudaSuccess) return e;
  dim3 grid((a.box_x1 - a.box_x0 + TX) / TX, (a.box_y1 - a.box_y0 + TY) / TY);
  k_interior<2, false><<<grid, NT, interior_smem_bytes(), s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_fill(double* p, double v, size_t n, cudaStream_t s) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  k_fill<<<blocks, 256, 0, s>>>(p, v, n);
  return cudaGetLastError();
}

// ghost frame (rows and columns within BC of an edge, 4 planes) of src
// into d1 and d2
__global__ void k_copy_frame(const double* __restrict__ src, double* __restrict__ d1,
                             double* __restrict__ d2, Field f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= frame_cells(f)) return;
  const size_t o = frame_offset(f, i);
  const double q = src[o];
  d1[o] = q;
  d2[o] = q;
}

cudaError_t launch_copy_frame(const double* src, double* d1, double* d2, const Field& f,
                              cudaStream_t s) {
  const int n = frame_cells(f);
  k_copy_frame<<<(n + 255) / 256, 256, 0, s>>>(src, d1, d2, f);
  return cudaGetLastError();
}

cudaError_t launch_periodic_ghosts(double* u, const Field& f, cudaStream_t s) {
  dim3 grid((f.nx + 127) / 128, f.ny);
  k_periodic_ghosts<<<grid, 128, 0, s>>>(u, f);
  return cudaGetLastError();
}

cudaError_t launch_cfl_max(const double* u, const Field& f, const DimConst& k, double* out,
                           cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  k_cfl_max<<<148 * 4, 256, 0, s>>>(u, f, k, reinterpret_cast<unsigned long long*>(out));
  return cudaGetLastError();
}

}  // namespace dim2d
