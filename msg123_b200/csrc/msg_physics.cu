// msg_physics.cu -- constitutive law, residual and Jacobian assembly on the
// structured 7-point cell stencil (B200, sm_100a).
//
// Layout in HBM (structure of arrays, reference local cell order i = ix + nx*(iy + ny*iz),
// iz = 0 is the top layer):
//   per cell   : h, kr, S (double), five real(SP) soil parameters (float)
//   per face   : hy[d*N + i], ab[d*N + i] for the up (d=0), north (1) and west (2) face
//                of cell i; the down/south/east faces of i are the up/north/west faces
//                of i+nx*ny, i+nx, i+1 (the reference's sat_hydf is symmetric bit for bit)
//   Jacobian   : dmat[N] and lu[d*N + i] for d = up..down, zero where no neighbour
// Each thread owns one cell; the six neighbours of a warp's cells are contiguous
// (x), one row apart (y) or one layer apart (z), so neighbour reads hit L1/L2.
#include "msg_ctx.cuh"
#include <vector>
#include <cstring>

namespace msg {

struct Geo {
  int nx, ny, nz, nxy, N;
};

__device__ __forceinline__ void cell_ijk(const Geo &g, int i, int &ix, int &iy, int &iz) {
  iz = i / g.nxy;
  int rem = i - iz * g.nxy;
  iy = rem / g.nx;
  ix = rem - iy * g.nx;
}

// set_sat_hyd (Set_condition.f90:2117-2139), interior face
__device__ __forceinline__ double sat_hyd(double hyd_c1, double hyd_c2, double d1, double d2) {
  double d12 = __dadd_rn(d1, d2);
  double c1 = __dmul_rn(hyd_c1, d12);
  double c2 = __dmul_rn(hyd_c2, d12);
  double cd12 = __dadd_rn(__dmul_rn(d1, c2), __dmul_rn(d2, c1));
  double cd = __ddiv_rn(1.0, cd12);
  return __dmul_rn(__dmul_rn(c1, c2), cd);
}

// ---------------------------------------------------------------------------------
// Face coefficients (set_connect / set_dis_adj / set_sat_hyd / set_chabyd,
// Set_condition.f90:1584-2158) in DIA form, plus the top and bottom layer arrays.
// ---------------------------------------------------------------------------------
__global__ void k_faces(Geo g, int sea_top, int free_drainage, const float *__restrict__ ksx,
                        const float *__restrict__ ksy, const float *__restrict__ ksz,
                        const double *__restrict__ dis, const double *__restrict__ far,
                        double *hy, double *ab, double *hydf_surf, double *abyd_surf,
                        double *sea_hydf, double *sea_abyd, double *drain, double *invd, double *top_invd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  cell_ijk(g, i, ix, iy, iz);
  const size_t N = g.N;
  // up
  if (iz > 0) {
    int nb = i - g.nxy;
    double d1 = dis[0 * N + i], d2 = dis[5 * N + nb];
    hy[0 * N + i] = sat_hyd((double)ksz[i], (double)ksz[nb], d1, d2);
    ab[0 * N + i] = __ddiv_rn(far[0 * N + i], __dadd_rn(d1, d2));
    invd[0 * N + i] = __ddiv_rn(1.0, __dadd_rn(d1, d2));
  } else {
    hy[0 * N + i] = 0.0; ab[0 * N + i] = 0.0; invd[0 * N + i] = 0.0;
    int s = i;
    double d1 = dis[0 * N + i];
    // sea face (dis12 = d1) and surface term (surf_elev - cell_cent = d1) share 1/d1
    top_invd[s] = __ddiv_rn(1.0, d1);
    if (sea_top) {
      sea_hydf[s] = (double)ksz[i];                       // bf == 1: hydf = tks
      sea_abyd[s] = __ddiv_rn(far[0 * N + i], d1);        // dis12 = d1
      hydf_surf[s] = 0.0;
      abyd_surf[s] = __ddiv_rn(0.0, d1);                  // surf_area stays 0 below a sea cell
    } else {
      sea_hydf[s] = 0.0; sea_abyd[s] = 0.0;
      hydf_surf[s] = (double)ksz[i];
      abyd_surf[s] = __ddiv_rn(far[0 * N + i], d1);       // surf_area / surf_dis
    }
  }
  // north
  if (iy > 0) {
    int nb = i - g.nx;
    double d1 = dis[1 * N + i], d2 = dis[4 * N + nb];
    hy[1 * N + i] = sat_hyd((double)ksy[i], (double)ksy[nb], d1, d2);
    ab[1 * N + i] = __ddiv_rn(far[1 * N + i], __dadd_rn(d1, d2));
    invd[1 * N + i] = __ddiv_rn(1.0, __dadd_rn(d1, d2));
  } else {
    hy[1 * N + i] = 0.0; ab[1 * N + i] = 0.0; invd[1 * N + i] = 0.0;
  }
  // west
  if (ix > 0) {
    int nb = i - 1;
    double d1 = dis[2 * N + i], d2 = dis[3 * N + nb];
    hy[2 * N + i] = sat_hyd((double)ksx[i], (double)ksx[nb], d1, d2);
    ab[2 * N + i] = __ddiv_rn(far[2 * N + i], __dadd_rn(d1, d2));
    invd[2 * N + i] = __ddiv_rn(1.0, __dadd_rn(d1, d2));
  } else {
    hy[2 * N + i] = 0.0; ab[2 * N + i] = 0.0; invd[2 * N + i] = 0.0;
  }
  if (iz == g.nz - 1) {
    int s = i - (g.nz - 1) * g.nxy;
    drain[s] = free_drainage ? __dmul_rn((double)ksz[i], far[5 * N + i]) : 0.0;
  }
}

// Reference CSR (off_index / off_row / conn_dir / left_off / right_off, plus the
// per-entry sat_hydf and area_dis computed from the row's own side).
__device__ __forceinline__ int row_count(const Geo &g, int i, int &nleft) {
  int ix, iy, iz;
  cell_ijk(g, i, ix, iy, iz);
  nleft = (iz > 0) + (iy > 0) + (ix > 0);
  return nleft + (ix < g.nx - 1) + (iy < g.ny - 1) + (iz < g.nz - 1);
}

__global__ void k_csr_count(Geo g, int *cnt, int *lcnt, int *rcnt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int nl;
  int c = row_count(g, i, nl);
  cnt[i] = c; lcnt[i] = nl; rcnt[i] = c - nl;
}

__global__ void k_csr_fill(Geo g, const int *offind, const int *lscan, const int *rscan,
                           const float *__restrict__ ksx, const float *__restrict__ ksy,
                           const float *__restrict__ ksz, const double *__restrict__ dis,
                           const double *__restrict__ far, int *offrow, int *conn_dir, int *left_off,
                           int *right_off, double *hydf, double *abyd) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  cell_ijk(g, i, ix, iy, iz);
  const size_t N = g.N;
  int k = offind[i], ln = lscan[i], rn = rscan[i];
  const int nbd[6] = {-g.nxy, -g.nx, -1, 1, g.nx, g.nxy};
  const bool has[6] = {iz > 0, iy > 0, ix > 0, ix < g.nx - 1, iy < g.ny - 1, iz < g.nz - 1};
  const float *kk[6] = {ksz, ksy, ksx, ksx, ksy, ksz};
  for (int d = 0; d < 6; ++d) {
    if (!has[d]) continue;
    int nb = i + nbd[d];
    offrow[k] = nb + 1;
    conn_dir[k] = d + 1;
    if (d < 3) { left_off[k] = ++ln; right_off[k] = 0; }
    else { right_off[k] = ++rn; left_off[k] = 0; }
    double d1 = dis[d * N + i], d2 = dis[(5 - d) * N + nb];
    hydf[k] = sat_hyd((double)kk[d][i], (double)kk[d][nb], d1, d2);
    abyd[k] = __ddiv_rn(far[d * N + i], __dadd_rn(d1, d2));
    ++k;
  }
}

// ---------------------------------------------------------------------------------
// calc_srat_rperm (Calc_parameter.f90:15-77), one cell.
// ---------------------------------------------------------------------------------
struct VG {
  double S, kr, alp;
};

// FORM 0 evaluates Mualem's kr = Se^(1/2) (1 - (1 - Se^(1/m))^m)^2 as the reference writes
// it.  FORM 1 evaluates the same function with two of its four pow calls replaced by
// identities of the van Genuchten curve: Se = (1 + beta)^-m, so Se^(1/m) = 1/(1 + beta) and
// (1 - Se^(1/m))^m = (beta / (1 + beta))^m = Se * beta^m, with beta^m = a^(n m) = a^(n-1)
// = beta / a (a = alpha |h|, n m = n - 1).  S is the same in both forms; kr differs by
// rounding (relative 1e-15 where kr is near 1, growing as 1e-16 / (1 - Se beta / a) in dry
// cells, where both forms cancel).  The limits agree: beta = 0 gives t = 1, Se = 0 gives
// kr = 0.
template <int FORM = 0>
__device__ __forceinline__ VG vg_eval(double pres, double top, double pertur, float reta, float retn,
                                      float resi, float poro, float ss) {
  VG o;
  double per_phead = __dadd_rn(__dsub_rn(pres, top), pertur);
  if (per_phead < 0.0) {
    double rn = (double)retn;
    double retm = __dsub_rn(1.0, __ddiv_rn(1.0, rn));
    double a = fabs(__dmul_rn(per_phead, (double)reta));
    double beta = pow(a, rn);
    double se = pow(__dadd_rn(1.0, beta), -retm);
    double theta = __dadd_rn((double)resi, __dmul_rn((double)(poro - resi), se));
    o.S = __ddiv_rn(theta, (double)poro);
    double t;
    if (FORM == 0) {
      t = __dsub_rn(1.0, pow(__dsub_rn(1.0, pow(se, __ddiv_rn(1.0, retm))), retm));
    } else {
      double ym = (beta == 0.0 || se == 0.0) ? 0.0 : __dmul_rn(se, __ddiv_rn(beta, a));
      t = __dsub_rn(1.0, ym);
    }
    o.kr = __dmul_rn(sqrt(se), __dmul_rn(t, t));
    o.alp = 0.0;
  } else {
    o.S = 1.0;
    o.kr = 1.0;
    o.alp = (double)ss;
  }
  return o;
}

template <int FORM>
__global__ void k_srat_rperm(int N, const double *__restrict__ h, double pertur, const double *__restrict__ top,
                             const float *__restrict__ reta, const float *__restrict__ retn,
                             const float *__restrict__ resi, const float *__restrict__ poro,
                             const float *__restrict__ ss, double *srat, double *kr, double *alp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  VG v = vg_eval<FORM>(h[i], top[i], pertur, reta[i], retn[i], resi[i], poro[i], ss[i]);
  srat[i] = v.S;
  kr[i] = v.kr;
  if (alp) alp[i] = v.alp;
}

// Storage part of calc_func (func_stochn, Calc_function.f90:176-210, with alp_old = alp_new
// as calc_func passes it) and, when asm_ is set, of make_matrix (form_stochn,
// Make_linearsystem.f90:148-193) with the perturbed evaluation at h + newper.
struct CellArgs {
  const double *h, *top, *vol, *h_old, *s_old;
  const float *reta, *retn, *resi, *poro, *ss;
  double delt_inv, newper, newper_inv;
  double *srat, *kr, *kr_per, *sto, *stod;
};

// ASM = false: calc_func's pass; ASM = true: make_matvec's pass.  REUSE (with ASM): S, kr
// and the storage term at h are already in srat / kr / sto from a residual evaluation at
// the same h (the previous Newton iteration ends with one), so only the perturbed
// evaluation at h + newper is made -- the same values bit for bit, half the pow calls.
template <bool ASM, bool REUSE = false, int FORM = 0>
__global__ void k_cell(int N, CellArgs a) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double hi = a.h[i], top = a.top[i];
  float reta = a.reta[i], retn = a.retn[i], resi = a.resi[i], poro = a.poro[i], ss = a.ss[i];
  if (REUSE) {
    VG v;
    v.S = a.srat[i];
    v.alp = (__dsub_rn(hi, top) < 0.0) ? 0.0 : (double)ss;   // vg_eval's branch at pertur = 0
    VG w = vg_eval<FORM>(hi, top, a.newper, reta, retn, resi, poro, ss);
    a.kr_per[i] = w.kr;
    double deri_srat = __dmul_rn(__dsub_rn(w.S, v.S), a.newper_inv);
    double deri_stor = __dmul_rn(__dmul_rn(v.alp, deri_srat), hi);
    double x = __dadd_rn(__dadd_rn(__dmul_rn((double)poro, deri_srat), __dmul_rn(v.alp, v.S)), deri_stor);
    a.stod[i] = __dmul_rn(__dmul_rn(-x, a.delt_inv), a.vol[i]);
    return;
  }
  VG v = vg_eval<FORM>(hi, top, 0.0, reta, retn, resi, poro, ss);
  double vol = a.vol[i];
  double ch1 = __dmul_rn(__dmul_rn(v.alp, a.s_old[i]), a.h_old[i]);
  double ch2 = __dmul_rn(__dmul_rn(v.alp, v.S), hi);
  double ch = __dadd_rn(__dsub_rn(ch2, ch1), __dmul_rn((double)poro, __dsub_rn(v.S, a.s_old[i])));
  a.sto[i] = __dmul_rn(__dmul_rn(-ch, a.delt_inv), vol);
  a.srat[i] = v.S;
  a.kr[i] = v.kr;
  if (ASM) {
    VG w = vg_eval<FORM>(hi, top, a.newper, reta, retn, resi, poro, ss);
    a.kr_per[i] = w.kr;
    double deri_srat = __dmul_rn(__dsub_rn(w.S, v.S), a.newper_inv);
    double deri_stor = __dmul_rn(__dmul_rn(v.alp, deri_srat), hi);
    double x = __dadd_rn(__dadd_rn(__dmul_rn((double)poro, deri_srat), __dmul_rn(v.alp, v.S)), deri_stor);
    a.stod[i] = __dmul_rn(__dmul_rn(-x, a.delt_inv), vol);
  }
}

// ---------------------------------------------------------------------------------
// Flux part of calc_func / make_matrix: func_connflow, func_rechterm, func_surfterm,
// func_sealterm (Calc_function.f90:212-513) and form_connflow, set_surfbound,
// set_seabound (Make_linearsystem.f90:195-285, :410-547), fused per cell.
// ---------------------------------------------------------------------------------
struct FluxArgs {
  Geo g;
  int sea_top, free_drainage;
  const double *h, *kr, *kr_per, *sto, *stod, *hy, *ab;
  const double *surf_top, *surf_bott, *surf_reli, *surf_parm, *hydf_surf, *abyd_surf, *surf_head;
  const double *calc_rech, *sea_hydf, *sea_abyd, *read_seal, *drain;
  const double *riv, *lak;    // [3S] stage, bed, area/distance per surface cell (nullable: none)
  const double *calc_well;    // [N] well rates of the time step (nullable: no wells)
  double newper, newper_inv;
  double *F;          // residual (calc_func) or rhs = -F (make_matvec)
  double *dmat, *lu;  // assembly outputs
  float *dmat_f, *lu_f;   // FP32 images for the mixed-precision V-cycle (nullable)
  double *part;       // partial sums of F^2 (nullable)
};

// func_surfterm for one top cell; returns the term and the Jacobian delh/over pair.
__device__ __forceinline__ double surf_term(double infs, double insh, double top, double bott, double reli,
                                            double parm, double hydf, double abyd, double kri, double &delh_out,
                                            double &over_out) {
  double delh, rati = 1.0, over;
  if (infs >= top) {
    delh = (insh > top) ? __dsub_rn(insh, infs) : __dsub_rn(top, infs);
    over = 1.0;
  } else if (infs >= bott) {
    delh = (insh > bott) ? __dsub_rn(insh, infs) : __dsub_rn(bott, infs);
    if (reli != 0.0) {
      double e = __ddiv_rn(__dsub_rn(infs, bott), reli);
      if (e > 1.0) e = 1.0;
      rati = pow(e, parm);
    }
    over = 1.0;
  } else if (insh > bott) {
    delh = __dsub_rn(insh, bott);
    if (reli != 0.0) {
      double e = __ddiv_rn(__dsub_rn(insh, bott), reli);
      if (e > 1.0) e = 1.0;
      rati = pow(e, parm);
    }
    over = 0.0;
  } else {
    delh = 0.0;
    over = 1.0;
  }
  delh_out = delh;
  over_out = over;
  return __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(hydf, abyd), delh), kri), rati);
}

// func_riveterm / func_laketerm (Calc_function.f90:393-473) for one surface cell s with
// stage/bed/abyd in st[s], st[S + s], st[2S + s] (abyd 0 where the cell has none, which
// makes both the term and its derivative an exact zero), and, for the assembly,
// set_rivebound / set_lakebound (Make_linearsystem.f90:287-408): -tran kr plus the chord of
// kr over newper times the head difference while the head is at or above the bed.
__device__ __forceinline__ double stage_term(const double *st, int S, int s, double infs, double hydf, double kri,
                                             double krpi, double newper_inv, bool asm_, double &dmat_out) {
  const double head = st[s], bott = st[S + s], abyd = st[2 * S + s];
  double delh, over;
  if (infs >= bott) { delh = __dsub_rn(head, infs); over = 1.0; }
  else if (head > bott) { delh = __dsub_rn(head, bott); over = 0.0; }
  else { delh = 0.0; over = 1.0; }
  if (asm_) {
    double tran = __dmul_rn(hydf, abyd);
    double deri = __dmul_rn(-tran, kri);
    double deri_ks = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dsub_rn(krpi, kri), newper_inv), delh), tran), over);
    dmat_out = __dadd_rn(deri, deri_ks);
  }
  return __dmul_rn(__dmul_rn(__dmul_rn(hydf, abyd), delh), kri);
}

// The flux passes run on a 3D grid of 256-thread blocks, each a 32 (x) by 8 (y) tile of one
// layer (blockIdx.z), so a cell's grid coordinates come from its block and lane with no
// integer division; flux_parts(c) is the number of blocks (one F^2 partial each).
template <bool ASM>
__device__ __forceinline__ void flux_body(const FluxArgs &a, double *sh) {
  const Geo g = a.g;
  const int ix = blockIdx.x * 32 + (threadIdx.x & 31), iy = blockIdx.y * 8 + (threadIdx.x >> 5), iz = blockIdx.z;
  double f2 = 0.0;
  if (ix < g.nx && iy < g.ny) {
    const size_t N = g.N;
    const int i = ix + g.nx * (iy + g.ny * iz);
    const double hi = a.h[i], kri = a.kr[i];
    const double krpi = ASM ? a.kr_per[i] : 0.0;
    const int nbd[6] = {-g.nxy, -g.nx, -1, 1, g.nx, g.nxy};
    const bool has[6] = {iz > 0, iy > 0, ix > 0, ix < g.nx - 1, iy < g.ny - 1, iz < g.nz - 1};
    double cf = 0.0, dc = 0.0;
#pragma unroll
    for (int d = 0; d < 6; ++d) {
      double luv = 0.0;
      if (has[d]) {
        int j = i + nbd[d];
        // face index: own up/north/west face, or the neighbour's for down/south/east
        size_t fi = (d < 3) ? (size_t)d * N + i : (size_t)(5 - d) * N + j;
        double hyd = a.hy[fi], abd = a.ab[fi];
        double hj = a.h[j], krj = a.kr[j];
        double delhead = __dsub_rn(hj, hi);
        double relat = upwind(-delhead, kri, krj);
        if (!ASM) {
          cf = __dadd_rn(cf, __dmul_rn(__dmul_rn(__dmul_rn(hyd, relat), abd), delhead));
        } else {
          double rel_hyd = __dmul_rn(hyd, relat);
          cf = __dadd_rn(cf, __dmul_rn(__dmul_rn(rel_hyd, abd), delhead));
          double deri_dcon = __dmul_rn(-rel_hyd, abd);
          double deri_lucon = __dmul_rn(rel_hyd, abd);
          double krpj = a.kr_per[j];
          double deri_hyd1 = __dmul_rn(hyd, upwind(__dadd_rn(-delhead, a.newper), krpi, krj));
          double deri_hyd2 = __dmul_rn(hyd, upwind(__dsub_rn(-delhead, a.newper), kri, krpj));
          double c1 = __dmul_rn(__dmul_rn(__dmul_rn(__dsub_rn(deri_hyd1, rel_hyd), a.newper_inv), delhead), abd);
          double c2 = __dmul_rn(__dmul_rn(__dmul_rn(__dsub_rn(deri_hyd2, rel_hyd), a.newper_inv), delhead), abd);
          luv = __dadd_rn(deri_lucon, c2);
          dc = __dadd_rn(__dadd_rn(dc, deri_dcon), c1);
        }
      }
      if (ASM) {
        a.lu[(size_t)d * N + i] = luv;
        if (a.lu_f) a.lu_f[(size_t)d * N + i] = (float)luv;
      }
    }
    // boundary terms of the top layer
    double fs = 0.0, ds = 0.0, sea = 0.0, sead = 0.0;
    if (iz == 0) {
      int s = i;
      double delh, over;
      double sf = surf_term(hi, a.surf_head[s], a.surf_top[s], a.surf_bott[s], a.surf_reli[s], a.surf_parm[s],
                            a.hydf_surf[s], a.abyd_surf[s], kri, delh, over);
      // funcvs = recf + surf + rivf + lakf (Calc_function.f90:86-90); dmats = surd + rivd + lakd
      double rv = 0.0, lk = 0.0, rvd = 0.0, lkd = 0.0;
      if (a.riv) rv = stage_term(a.riv, g.nxy, s, hi, a.hydf_surf[s], kri, krpi, a.newper_inv, ASM, rvd);
      if (a.lak) lk = stage_term(a.lak, g.nxy, s, hi, a.hydf_surf[s], kri, krpi, a.newper_inv, ASM, lkd);
      fs = __dadd_rn(__dadd_rn(__dadd_rn(a.calc_rech[s], sf), rv), lk);
      if (ASM) {
        double tran = __dmul_rn(a.hydf_surf[s], a.abyd_surf[s]);
        double deri_s = __dmul_rn(-tran, kri);
        double deri_ks = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(__dsub_rn(krpi, kri), a.newper_inv), delh), tran), over);
        ds = __dadd_rn(__dadd_rn(__dadd_rn(deri_s, deri_ks), rvd), lkd);
      }
      if (a.sea_top) {
        double delhs = __dsub_rn(a.read_seal[s], hi);
        sea = __dmul_rn(__dmul_rn(__dmul_rn(a.sea_hydf[s], kri), a.sea_abyd[s]), delhs);
        if (ASM) {
          double per_sea = __dmul_rn(krpi, a.sea_hydf[s]);
          double rel_sea = __dmul_rn(kri, a.sea_hydf[s]);
          double deri_sea = __dmul_rn(-rel_sea, a.sea_abyd[s]);
          double deri_ks = __dmul_rn(__dmul_rn(__dmul_rn(__dsub_rn(per_sea, rel_sea), a.newper_inv), delhs), a.sea_abyd[s]);
          sead = __dadd_rn(deri_sea, deri_ks);
        }
      }
    }
    // funcv = funcvs + stof + conf + welf + seaf (Calc_function.f90:92-96)
    const double wel = a.calc_well ? a.calc_well[i] : 0.0;
    double f = __dadd_rn(__dadd_rn(__dadd_rn(__dadd_rn(fs, a.sto[i]), cf), wel), sea);
    double dd = 0.0;
    if (ASM) dd = __dadd_rn(__dadd_rn(__dadd_rn(ds, a.stod[i]), dc), sead);
    if (a.free_drainage && iz == g.nz - 1) {
      double coef = a.drain[i - (g.nz - 1) * g.nxy];
      if (coef != 0.0) {
        f = __dadd_rn(f, -__dmul_rn(coef, kri));
        if (ASM) dd = __dadd_rn(dd, -__dmul_rn(__dmul_rn(__dsub_rn(krpi, kri), a.newper_inv), coef));
      }
    }
    if (ASM) {
      a.F[i] = -f;
      a.dmat[i] = dd;
      if (a.dmat_f) a.dmat_f[i] = (float)dd;
    } else {
      a.F[i] = f;
    }
    f2 = __dmul_rn(f, f);
  }
  if (a.part) {
    double s = block_sum<256>(f2, sh);
    if (threadIdx.x == 0) a.part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = s;
  }
}

// Residual pass: at most 48 registers so that five 256-thread blocks stay resident per SM
// (the pass is bound by the latency of its 27 loads per cell, not by bandwidth).
__global__ void __launch_bounds__(256, 5) k_flux_res(FluxArgs a) {
  __shared__ double sh[8];
  flux_body<false>(a, sh);
}

// Assembly pass (residual + Jacobian rows).
__global__ void __launch_bounds__(256) k_flux_asm(FluxArgs a) {
  __shared__ double sh[8];
  flux_body<true>(a, sh);
}

// DIA -> reference CSR order export of lumat.
__global__ void k_dia_to_csr(Geo g, const int *offind, const double *lu, double *lumat) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  int ix, iy, iz;
  cell_ijk(g, i, ix, iy, iz);
  const bool has[6] = {iz > 0, iy > 0, ix > 0, ix < g.nx - 1, iy < g.ny - 1, iz < g.nz - 1};
  int k = offind[i];
  for (int d = 0; d < 6; ++d)
    if (has[d]) lumat[k++] = lu[(size_t)d * g.N + i];
}

// calc_mass (Calc_function.f90:103-174) terms of cell i, each times delt: acc[0] storage
// (func_stochn), acc[1] flow from the neighbours in CSR face order (func_connflow),
// acc[2] recharge (func_rechterm), acc[3] surface (func_surfterm with surf_old), acc[4] sea
// (func_sealterm: one sea face per top cell), acc[5] free drainage (extension), acc[6] wells
// (func_wellterm), acc[7] rivers, acc[8] lakes.  acc[2..4], acc[7], acc[8] belong to top
// cells, acc[5] to bottom cells; the others are zero.
__device__ __forceinline__ void mass_terms(const FluxArgs &a, int i, const double *h_old, const double *s_old,
                                           const double *s_new, const double *alp_new, const double *alp_old,
                                           const float *poro, const double *vol, double delt_inv, double delt,
                                           double acc[9]) {
  const Geo g = a.g;
  for (int q = 0; q < 9; ++q) acc[q] = 0.0;
  int ix, iy, iz;
  cell_ijk(g, i, ix, iy, iz);
  double hi = a.h[i], kri = a.kr[i];
  double ch1 = __dmul_rn(__dmul_rn(alp_old[i], s_old[i]), h_old[i]);
  double ch2 = __dmul_rn(__dmul_rn(alp_new[i], s_new[i]), hi);
  double ch = __dadd_rn(__dsub_rn(ch2, ch1), __dmul_rn((double)poro[i], __dsub_rn(s_new[i], s_old[i])));
  acc[0] = __dmul_rn(__dmul_rn(__dmul_rn(-ch, delt_inv), vol[i]), delt);
  const int nbd[6] = {-g.nxy, -g.nx, -1, 1, g.nx, g.nxy};
  const bool has[6] = {iz > 0, iy > 0, ix > 0, ix < g.nx - 1, iy < g.ny - 1, iz < g.nz - 1};
  double cf = 0.0;
  for (int d = 0; d < 6; ++d) {
    if (!has[d]) continue;
    int j = i + nbd[d];
    size_t fi = (d < 3) ? (size_t)d * g.N + i : (size_t)(5 - d) * g.N + j;
    double delhead = __dsub_rn(a.h[j], hi);
    double relat = upwind(-delhead, kri, a.kr[j]);
    cf = __dadd_rn(cf, __dmul_rn(__dmul_rn(__dmul_rn(a.hy[fi], relat), a.ab[fi]), delhead));
  }
  acc[1] = __dmul_rn(cf, delt);
  if (a.calc_well) acc[6] = __dmul_rn(a.calc_well[i], delt);
  if (iz == 0) {
    double delh, over, dummy;
    double sf = surf_term(hi, a.surf_head[i], a.surf_top[i], a.surf_bott[i], a.surf_reli[i], a.surf_parm[i],
                          a.hydf_surf[i], a.abyd_surf[i], kri, delh, over);
    acc[2] = __dmul_rn(a.calc_rech[i], delt);
    acc[3] = __dmul_rn(sf, delt);
    if (a.riv) acc[7] = __dmul_rn(stage_term(a.riv, g.nxy, i, hi, a.hydf_surf[i], kri, 0.0, 0.0, false, dummy), delt);
    if (a.lak) acc[8] = __dmul_rn(stage_term(a.lak, g.nxy, i, hi, a.hydf_surf[i], kri, 0.0, 0.0, false, dummy), delt);
    if (a.sea_top)
      acc[4] = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(a.sea_hydf[i], kri), a.sea_abyd[i]), __dsub_rn(a.read_seal[i], hi)), delt);
  }
  if (a.free_drainage && iz == g.nz - 1) {
    double coef = a.drain[i - (g.nz - 1) * g.nxy];
    acc[5] = __dmul_rn(-__dmul_rn(coef, kri), delt);
  }
}

// calc_mass summed over cells: block partial sums of the six terms.
__global__ void __launch_bounds__(256) k_mass(FluxArgs a, const double *h_old, const double *s_old,
                                              const double *s_new, const double *alp_new, const double *alp_old,
                                              const float *poro, const double *vol, double delt_inv, double delt,
                                              double *part9) {
  __shared__ double sh[8];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (i < a.g.N) mass_terms(a, i, h_old, s_old, s_new, alp_new, alp_old, poro, vol, delt_inv, delt, acc);
  for (int q = 0; q < 9; ++q) {
    double s = block_sum<256>(acc[q], sh);
    if (threadIdx.x == 0) part9[(size_t)q * gridDim.x + blockIdx.x] = s;
  }
}

// calc_cell_mas (Calc_output.f90:54-91): the same terms per cell, in the reference's
// arrays -- storage, flow, sea and wells per cell [N]; recharge, surface, river, lake and
// drainage per surface column [S] (drainage leaves through the column's bottom cell).
__global__ void __launch_bounds__(256) k_cell_mass(FluxArgs a, const double *h_old, const double *s_old,
                                                   const double *s_new, const double *alp_new,
                                                   const double *alp_old, const float *poro, const double *vol,
                                                   double delt_inv, double delt, double *sto, double *con,
                                                   double *sea, double *wel, double *rec, double *sur, double *riv,
                                                   double *lak, double *drn) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.g.N) return;
  double acc[9];
  mass_terms(a, i, h_old, s_old, s_new, alp_new, alp_old, poro, vol, delt_inv, delt, acc);
  sto[i] = acc[0];
  con[i] = acc[1];
  sea[i] = acc[4];
  wel[i] = acc[6];
  if (i < a.g.nxy) { rec[i] = acc[2]; sur[i] = acc[3]; riv[i] = acc[7]; lak[i] = acc[8]; }
  if (i >= (a.g.nz - 1) * a.g.nxy) drn[i - (a.g.nz - 1) * a.g.nxy] = acc[5];
}

// calc_outvelc (Calc_output.f90:168-241) for cell i: the Darcy velocity through each face
// (face-major facev[d*N + i], d = up, north, west, east, south, down): regular faces
// hydf * relat * delhead * (1/dis12) in the reference's product order; the top face the
// sea term (sea layer above) or else the surface term, both with 1/dis2face(up); the bottom
// face of the lowest layer the unit-gradient velocity -Ksz kr under free drainage (an
// extension); faces with no connection 0.  Then the cell-centred components pointv[c*N + i]
// (c = x, y, z) from the opposite face pairs: half the difference where the two velocities
// have opposite signs, the whole difference otherwise, z negated (upward positive).
__global__ void __launch_bounds__(256) k_velocity(FluxArgs a, const double *invd, const double *top_invd,
                                                  const float *ksz, double *facev, double *pointv) {
  const Geo g = a.g;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.N) return;
  const size_t N = g.N;
  int ix, iy, iz;
  cell_ijk(g, i, ix, iy, iz);
  const double hi = a.h[i], kri = a.kr[i];
  const int nbd[6] = {-g.nxy, -g.nx, -1, 1, g.nx, g.nxy};
  const bool has[6] = {iz > 0, iy > 0, ix > 0, ix < g.nx - 1, iy < g.ny - 1, iz < g.nz - 1};
  double fv[6];
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    fv[d] = 0.0;
    if (has[d]) {
      int j = i + nbd[d];
      size_t fi = (d < 3) ? (size_t)d * N + i : (size_t)(5 - d) * N + j;
      double delhead = __dsub_rn(a.h[j], hi);
      double relat = upwind(-delhead, kri, a.kr[j]);
      fv[d] = __dmul_rn(__dmul_rn(__dmul_rn(a.hy[fi], relat), delhead), invd[fi]);
    }
  }
  if (iz == 0) {
    if (a.sea_top) {
      double delhead = __dsub_rn(a.read_seal[i], hi);
      fv[0] = __dmul_rn(__dmul_rn(__dmul_rn(a.sea_hydf[i], delhead), top_invd[i]), kri);
    } else {
      double delhead = __dsub_rn(a.surf_head[i], hi);
      fv[0] = __dmul_rn(__dmul_rn(__dmul_rn(a.hydf_surf[i], delhead), top_invd[i]), kri);
    }
  }
  if (a.free_drainage && iz == g.nz - 1) fv[5] = -__dmul_rn((double)ksz[i], kri);
#pragma unroll
  for (int d = 0; d < 6; ++d) facev[(size_t)d * N + i] = fv[d];
#pragma unroll
  for (int d = 1; d <= 3; ++d) {
    double x = fv[d - 1], y = fv[6 - d], v;
    if ((x > 0.0 && y < 0.0) || (x < 0.0 && y > 0.0)) v = __dmul_rn(__dsub_rn(x, y), 0.5);
    else v = __dsub_rn(x, y);
    if (d == 1) v = -v;
    pointv[(size_t)(3 - d) * N + i] = v;
  }
}

// set_vwell_head (Time_module.f90:1137-1158: calc_vheadout / calc_vheadin, :1253-1335), one
// thread per well, connections in the reference's order: the head without pumping is the
// kr*abyd-weighted mean of the well's cell heads, the pumping rate over the total
// conductance raises it, and each cell where that head or the cell's own head is above
// the well bottom gets kr*abyd*(whead - head) (calc_well zeroed beforehand; a cell belongs
// to one well).  kr is evaluated at head_new, the state the reference's rel_perm holds there.
template <int FORM>
__global__ void k_wells(int nwell, const int *__restrict__ w_index, const int *__restrict__ w_conn,
                        const double *__restrict__ w_abyd, const double *__restrict__ w_bott,
                        const double *__restrict__ w_rate, CellArgs a, double *calc_well) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwell) return;
  double tot_cond = 0.0, tot_flux = 0.0, whead = 0.0;
  for (int k = w_index[w]; k < w_index[w + 1]; ++k) {
    int j = w_conn[k];
    double kr = vg_eval<FORM>(a.h[j], a.top[j], 0.0, a.reta[j], a.retn[j], a.resi[j], a.poro[j], a.ss[j]).kr;
    tot_cond = __dadd_rn(tot_cond, __dmul_rn(kr, w_abyd[k]));
    tot_flux = __dadd_rn(tot_flux, __dmul_rn(__dmul_rn(kr, w_abyd[k]), a.h[j]));
  }
  if (tot_cond == 0.0) return;
  whead = __ddiv_rn(tot_flux, tot_cond);
  whead = __dadd_rn(whead, __ddiv_rn(w_rate[w], tot_cond));
  for (int k = w_index[w]; k < w_index[w + 1]; ++k) {
    int j = w_conn[k];
    if (whead > w_bott[w] || a.h[j] > w_bott[w]) {
      double kr = vg_eval<FORM>(a.h[j], a.top[j], 0.0, a.reta[j], a.retn[j], a.resi[j], a.poro[j], a.ss[j]).kr;
      calc_well[j] = __dadd_rn(calc_well[j], __dmul_rn(__dmul_rn(kr, w_abyd[k]), __dsub_rn(whead, a.h[j])));
    }
  }
}

// ---------------------------------------------------------------------------------
// Host wrappers
// ---------------------------------------------------------------------------------
static Geo geo(const msg_ctx *c) { return Geo{c->nx, c->ny, c->nz, c->nxy, c->N}; }
static dim3 flux_grid(const msg_ctx *c) { return dim3((c->nx + 31) / 32, (c->ny + 7) / 8, c->nz); }
int flux_parts(const msg_ctx *c) {
  const dim3 g = flux_grid(c);
  return (int)(g.x * g.y * g.z);
}
static int nblk(int n) { return (n + kThreads - 1) / kThreads; }

int build_connectivity(msg_ctx *c, const msg_grid_t *g) {
  const size_t N = c->N;
  float *d_ksx = nullptr, *d_ksy = nullptr;
  double *d_dis = nullptr, *d_far = nullptr;
  MSG_CUDA(cudaMalloc(&d_ksx, N * 4));
  MSG_CUDA(cudaMalloc(&d_ksy, N * 4));
  MSG_CUDA(cudaMalloc(&d_dis, 6 * N * 8));
  MSG_CUDA(cudaMalloc(&d_far, 6 * N * 8));
  MSG_CUDA(cudaMemcpyAsync(d_ksx, g->ksx, N * 4, cudaMemcpyHostToDevice, c->stream));
  MSG_CUDA(cudaMemcpyAsync(d_ksy, g->ksy, N * 4, cudaMemcpyHostToDevice, c->stream));
  MSG_CUDA(cudaMemcpyAsync(d_dis, g->dis2face, 6 * N * 8, cudaMemcpyHostToDevice, c->stream));
  MSG_CUDA(cudaMemcpyAsync(d_far, g->face_area, 6 * N * 8, cudaMemcpyHostToDevice, c->stream));
  Geo gg = geo(c);
  k_faces<<<nblk(c->N), kThreads, 0, c->stream>>>(gg, c->sea_top, c->free_drainage, d_ksx, d_ksy, c->ksz, d_dis,
                                                     d_far, c->hy, c->ab, c->hydf_surf, c->abyd_surf, c->sea_hydf,
                                                     c->sea_abyd, c->drain, c->invd, c->top_invd);
  MSG_CHECK_LAUNCH();
  // CSR
  int *cnt, *lcnt, *rcnt, *lscan, *rscan;
  MSG_CUDA(cudaMalloc(&cnt, N * 4));
  MSG_CUDA(cudaMalloc(&lcnt, N * 4));
  MSG_CUDA(cudaMalloc(&rcnt, N * 4));
  MSG_CUDA(cudaMalloc(&lscan, N * 4));
  MSG_CUDA(cudaMalloc(&rscan, N * 4));
  k_csr_count<<<nblk(c->N), kThreads, 0, c->stream>>>(gg, cnt, lcnt, rcnt);
  MSG_CHECK_LAUNCH();
  int total = 0, tl = 0, tr = 0;
  int rc;
  if ((rc = scan_exclusive(c, cnt, c->offind, c->N, &total))) return rc;
  if ((rc = scan_exclusive(c, lcnt, lscan, c->N, &tl))) return rc;
  if ((rc = scan_exclusive(c, rcnt, rscan, c->N, &tr))) return rc;
  MSG_CUDA(cudaMemcpyAsync(c->offind + c->N, &total, 4, cudaMemcpyHostToDevice, c->stream));
  c->nnz = total;
  MSG_CUDA(cudaMalloc(&c->offrow, (size_t)total * 4));
  MSG_CUDA(cudaMalloc(&c->conn_dir, (size_t)total * 4));
  MSG_CUDA(cudaMalloc(&c->left_off, (size_t)total * 4));
  MSG_CUDA(cudaMalloc(&c->right_off, (size_t)total * 4));
  MSG_CUDA(cudaMalloc(&c->hydf_conn, (size_t)total * 8));
  MSG_CUDA(cudaMalloc(&c->abyd_conn, (size_t)total * 8));
  k_csr_fill<<<nblk(c->N), kThreads, 0, c->stream>>>(gg, c->offind, lscan, rscan, d_ksx, d_ksy, c->ksz, d_dis, d_far,
                                                      c->offrow, c->conn_dir, c->left_off, c->right_off,
                                                      c->hydf_conn, c->abyd_conn);
  MSG_CHECK_LAUNCH();
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(cnt); cudaFree(lcnt); cudaFree(rcnt); cudaFree(lscan); cudaFree(rscan);
  cudaFree(d_ksx); cudaFree(d_ksy); cudaFree(d_dis); cudaFree(d_far);
  return MSG_OK;
}

// calc_wtable (Calc_output.f90:20-52), one thread per surface column: walk up from the
// bottom layer, keep the head of each cell, stop at the first cell that is not fully
// saturated.  Layer k of column i is cell k * S + i (S = nx * ny cells per layer).
__global__ void k_water_table(int S, int nz, const double *__restrict__ h, const double *__restrict__ srat,
                              double *wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S) return;
  double w = 0.0;
  for (int k = nz - 1; k >= 0; --k) {
    const size_t cell = (size_t)k * S + i;
    w = h[cell];
    if (srat[cell] != 1.0) break;
  }
  wt[i] = w;
}

int launch_water_table(msg_ctx *c, double *wt) {
  k_water_table<<<nblk(c->S), kThreads, 0, c->stream>>>(c->S, c->nz, c->head_new, c->srat_new, wt);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int launch_srat_rperm(msg_ctx *c, const double *h, double pertur, double *srat, double *kr, double *alp) {
  auto k = c->prm.vg_form ? k_srat_rperm<1> : k_srat_rperm<0>;
  k<<<nblk(c->N), kThreads, 0, c->stream>>>(c->N, h, pertur, c->cell_top, c->reta, c->retn, c->resi, c->poro, c->ss,
                                            srat, kr, alp);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

static FluxArgs flux_args(msg_ctx *c, const double *h) {
  FluxArgs a;
  a.g = geo(c);
  a.sea_top = c->sea_top;
  a.free_drainage = c->free_drainage;
  a.h = h; a.kr = c->kr; a.kr_per = c->kr_per; a.sto = c->sto; a.stod = c->stod; a.hy = c->hy; a.ab = c->ab;
  a.surf_top = c->surf_top; a.surf_bott = c->surf_bott; a.surf_reli = c->surf_reli; a.surf_parm = c->surf_parm;
  a.hydf_surf = c->hydf_surf; a.abyd_surf = c->abyd_surf; a.surf_head = c->surf_head;
  a.calc_rech = c->calc_rech; a.sea_hydf = c->sea_hydf; a.sea_abyd = c->sea_abyd; a.read_seal = c->read_seal;
  a.drain = c->drain;
  a.riv = c->riv; a.lak = c->lak; a.calc_well = c->calc_well;
  a.newper = c->newper; a.newper_inv = c->newper_inv;
  a.F = nullptr; a.dmat = nullptr; a.lu = nullptr; a.part = nullptr;
  a.dmat_f = nullptr; a.lu_f = nullptr;
  return a;
}

static CellArgs cell_args(msg_ctx *c, const double *h) {
  CellArgs a;
  a.h = h; a.top = c->cell_top; a.vol = c->cell_vol; a.h_old = c->head_old; a.s_old = c->srat_old;
  a.reta = c->reta; a.retn = c->retn; a.resi = c->resi; a.poro = c->poro; a.ss = c->ss;
  a.delt_inv = c->delt_inv; a.newper = c->newper; a.newper_inv = c->newper_inv;
  a.srat = c->srat_new; a.kr = c->kr; a.kr_per = c->kr_per; a.sto = c->sto; a.stod = c->stod;
  return a;
}

int launch_calc_func(msg_ctx *c, const double *h, double *F, bool norm) {
  const int bc = c->blk_cell > 0 ? c->blk_cell : kThreads;
  auto k = c->prm.vg_form ? k_cell<false, false, 1> : k_cell<false, false, 0>;
  k<<<(c->N + bc - 1) / bc, bc, 0, c->stream>>>(c->N, cell_args(c, h));
  MSG_CHECK_LAUNCH();
  FluxArgs a = flux_args(c, h);
  a.F = F;
  a.part = norm ? c->part : nullptr;
  k_flux_res<<<flux_grid(c), 256, 0, c->stream>>>(a);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int launch_make_matvec(msg_ctx *c, bool reuse, double *rhs_out) {
  const int bc = c->blk_cell > 0 ? c->blk_cell : kThreads;
  auto k = c->prm.vg_form ? (reuse ? k_cell<true, true, 1> : k_cell<true, false, 1>)
                           : (reuse ? k_cell<true, true, 0> : k_cell<true, false, 0>);
  k<<<(c->N + bc - 1) / bc, bc, 0, c->stream>>>(c->N, cell_args(c, c->head_new));
  MSG_CHECK_LAUNCH();
  FluxArgs a = flux_args(c, c->head_new);
  a.F = rhs_out ? rhs_out : c->rhs;
  a.dmat = c->dmat;
  a.lu = c->lu;
  a.dmat_f = c->dmat_f;
  a.lu_f = c->lu_f;
  a.part = c->part;
  k_flux_asm<<<flux_grid(c), 256, 0, c->stream>>>(a);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int launch_dia_to_csr(msg_ctx *c, double *lumat_dev) {
  k_dia_to_csr<<<nblk(c->N), kThreads, 0, c->stream>>>(geo(c), c->offind, c->lu, lumat_dev);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int launch_mass(msg_ctx *c, double *out9_dev) {
  // old-level vG (alp_old) into tmpv / kr_per scratch, then new-level into srat_new / kr / alp
  double *alp_old = c->tmpv, *s_tmp = c->sto, *kr_tmp = c->kr_per;
  int rc;
  if ((rc = launch_srat_rperm(c, c->head_old, 0.0, s_tmp, kr_tmp, alp_old))) return rc;
  if ((rc = launch_srat_rperm(c, c->head_new, 0.0, c->srat_new, c->kr, c->alp))) return rc;
  FluxArgs a = flux_args(c, c->head_new);
  a.surf_head = c->surf_old;
  int nb = nblk(c->N);
  double *part9 = nullptr;
  MSG_CUDA(cudaMalloc(&part9, (size_t)9 * nb * 8));
  k_mass<<<nb, 256, 0, c->stream>>>(a, c->head_old, c->srat_old, c->srat_new, c->alp, alp_old, c->poro, c->cell_vol,
                                     c->delt_inv, c->delt, part9);
  MSG_CHECK_LAUNCH();
  std::vector<double> hp((size_t)9 * nb);
  MSG_CUDA(cudaMemcpyAsync(hp.data(), part9, hp.size() * 8, cudaMemcpyDeviceToHost, c->stream));
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  cudaFree(part9);
  double out[9] = {0};
  const int map[9] = {0, 1, 2, 4, 7, 8, 3, 5, 6};
  for (int q = 0; q < 9; ++q) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += hp[(size_t)q * nb + b];
    out[map[q]] = s;
  }
  MSG_CUDA(cudaMemcpyAsync(out9_dev, out, sizeof(out), cudaMemcpyHostToDevice, c->stream));
  MSG_CUDA(cudaStreamSynchronize(c->stream));
  return MSG_OK;
}

int launch_cell_mass(msg_ctx *c, double *sto, double *con, double *sea, double *wel, double *rec, double *sur,
                     double *riv, double *lak, double *drn) {
  // old-level vG (alp_old) into tmpv / kr_per scratch, then new-level into srat_new / kr / alp,
  // as launch_mass does
  double *alp_old = c->tmpv, *s_tmp = c->sto, *kr_tmp = c->kr_per;
  int rc;
  if ((rc = launch_srat_rperm(c, c->head_old, 0.0, s_tmp, kr_tmp, alp_old))) return rc;
  if ((rc = launch_srat_rperm(c, c->head_new, 0.0, c->srat_new, c->kr, c->alp))) return rc;
  FluxArgs a = flux_args(c, c->head_new);
  a.surf_head = c->surf_old;
  k_cell_mass<<<nblk(c->N), 256, 0, c->stream>>>(a, c->head_old, c->srat_old, c->srat_new, c->alp, alp_old, c->poro,
                                                  c->cell_vol, c->delt_inv, c->delt, sto, con, sea, wel, rec, sur,
                                                  riv, lak, drn);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int launch_velocity(msg_ctx *c, double *facev, double *pointv) {
  // rel_perm at head_new, as calc_outvelc reads it after the step
  int rc;
  if ((rc = launch_srat_rperm(c, c->head_new, 0.0, c->srat_new, c->kr, c->alp))) return rc;
  FluxArgs a = flux_args(c, c->head_new);
  k_velocity<<<nblk(c->N), 256, 0, c->stream>>>(a, c->invd, c->top_invd, c->ksz, facev, pointv);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

int launch_wells(msg_ctx *c) {
  if (!c->calc_well) return MSG_OK;
  MSG_CUDA(cudaMemsetAsync(c->calc_well, 0, (size_t)c->N * 8, c->stream));
  if (c->nwell <= 0) return MSG_OK;
  CellArgs a = cell_args(c, c->head_new);
  int nb = (c->nwell + 127) / 128;
  if (c->prm.vg_form) k_wells<1><<<nb, 128, 0, c->stream>>>(c->nwell, c->w_index, c->w_conn, c->w_abyd, c->w_bott,
                                                           c->w_rate, a, c->calc_well);
  else k_wells<0><<<nb, 128, 0, c->stream>>>(c->nwell, c->w_index, c->w_conn, c->w_abyd, c->w_bott, c->w_rate, a,
                                             c->calc_well);
  MSG_CHECK_LAUNCH();
  return MSG_OK;
}

}  // namespace msg
