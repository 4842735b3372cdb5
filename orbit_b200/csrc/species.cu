// K1b: species sink diagonals and source-coupling diagonals of one bin, and
// the coupled right-hand sides of the multi-species solve.
//
// Every species operator of the reference is L_s = T + diag(d_s) and every
// source coupling K[(target, source)] is a diagonal block
// (assemble_species_operators, orbit/core/operator.py:371-595), so the whole
// species-dependent part of the operators is per-cell arithmetic: one thread
// per cell reads the deposition, partitioning and chemistry fields and writes
// the 14 diagonals and the 6 coupling diagonals.  Formulas follow
//   assemble_deposition           orbit/core/deposition.py:101-146
//   _get_dry_dep_velocity_2d      orbit/core/deposition.py:263-304
//   _get_wet_dep_rate_3d          orbit/core/deposition.py:307-360
//   _get_soa_photolysis_rate_3d   orbit/core/deposition.py:149-168
//   _get_hno3_vd / _get_o3_vd     orbit/core/deposition.py:219-260
//   SO2 oxidation blocks          orbit/core/chemistry.py:13-47
//   NOx, O3, CO, VBS aging        orbit/core/operator.py:455-585
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"

namespace orbit {

// Species indices of the 14-species inventory (deposition.py:54-76).
enum {
  kVbsC100 = 0, kPm25 = 1, kTotalNh = 2, kSo2 = 3, kNox = 4, kPso4 = 5, kTotalNo3 = 6, kO3 = 7, kCo = 8,
  kVbsC10 = 9, kVbsC1 = 10, kVbsC01 = 11, kVbsC1000 = 12, kPoa = 13, kNumSpecies = 14
};

namespace {

// Position of a VBS species in the bin order C01, C1, C10, C100, C1000
// (IDX_VBS_BINS, deposition.py:84-85), -1 otherwise.
__device__ __forceinline__ int vbs_pos(int s) {
  switch (s) {
    case kVbsC01: return 0;
    case kVbsC1: return 1;
    case kVbsC10: return 2;
    case kVbsC100: return 3;
    case kVbsC1000: return 4;
    default: return -1;
  }
}

__global__ void k_species_diag(int nz, int ny, int nx, orbit_species_fields_t f, double* __restrict__ d,
                               double* __restrict__ ksrc) {
  const int64_t N = (int64_t)nz * ny * nx;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int64_t nxy = (int64_t)nx * ny;
  const int64_t s2 = c % nxy;  // surface cell of this column
  const bool surf = c < nxy;
  const double dz0 = f.Dz[s2];
  const double inv_dz0 = dz0 > 0.0 ? 1.0 / dz0 : 0.0;
  const double pw = f.particle_wet_dep[c];
  const double gw = f.other_gas_wet_dep[c];
  const double pd0 = f.particle_dry_dep[s2];
  for (int s = 0; s < kNumSpecies; ++s) {
    double wet = 0.0, vd = 0.0, extra = 0.0;
    const int vp = vbs_pos(s);
    if (vp >= 0) {
      wet = f.fp_vbs ? f.fp_vbs[(int64_t)vp * N + c] * pw : pw;
      if (surf) {
        if (f.fp_vbs_surface) {
          const double F = f.fp_vbs_surface[(int64_t)vp * nxy + s2];
          const double voc = f.voc_dry_dep ? f.voc_dry_dep[s2] : 1.0e-3;
          vd = F * pd0 + (1.0 - F) * voc;
        } else {
          vd = pd0;
        }
      }
      if (f.j_no2 && f.a_photo > 0.0)
        extra += f.a_photo * f.j_no2[c] * (f.fp_vbs ? f.fp_vbs[(int64_t)vp * N + c] : 1.0);
    } else if (s == kPm25 || s == kPoa || s == kPso4) {
      wet = pw;
      vd = pd0;
    } else if (s == kTotalNh) {
      const double p = f.nh_part[c];
      wet = (1.0 - p) * gw + p * pw;
      if (surf) {
        const double p0 = f.nh_part[s2];
        vd = (1.0 - p0) * f.nh3_dry_dep[s2] + p0 * pd0;
      }
    } else if (s == kSo2) {
      wet = f.so2_wet_dep[c];
      vd = f.so2_dry_dep[s2];
      if (f.so2_ox) extra += f.so2_ox[c];
    } else if (s == kNox) {
      vd = f.nox_dry_dep[s2];
      if (f.nox_ox) extra += f.nox_ox[c];
    } else if (s == kTotalNo3) {
      const double p = f.no3_part ? f.no3_part[c] : 0.0;
      wet = (1.0 - p) * gw + p * pw;
      if (surf) {
        const double p0 = f.no3_part ? f.no3_part[s2] : 0.0;
        const double vh = f.hno3_dry_dep ? f.hno3_dry_dep[s2] : 0.03;
        vd = (1.0 - p0) * vh + p0 * pd0;
      }
    } else if (s == kO3) {
      if (f.o3_dry_dep) vd = f.o3_dry_dep[s2];
      else vd = (f.is_land ? f.is_land[s2] > 0.0 : true) ? 0.004 : 0.0005;
      if (f.o3_loss) extra += f.o3_loss[c];
    } else if (s == kCo) {
      if (f.co_loss) extra += f.co_loss[c];
    }
    double rate = wet + extra;
    if (surf) rate += vd * inv_dz0;
    d[(int64_t)s * N + c] = rate;
  }
  // source couplings: pSO4 <- SO2, TotalNO3 <- NOx, then the aging cascade
  double k0 = f.so2_ox ? -f.so2_ox[c] : 0.0;
  double k1 = f.nox_ox ? -f.nox_ox[c] : 0.0;
  double kag[4] = {0.0, 0.0, 0.0, 0.0};
  if (f.archive_oh) {
    const double roh = f.k_age * f.archive_oh[c];
    const int src[4] = {kVbsC1000, kVbsC100, kVbsC10, kVbsC1};
    for (int q = 0; q < 4; ++q) {
      double r = roh;
      if (f.fp_vbs) {
        const double F = fmin(fmax(f.fp_vbs[(int64_t)vbs_pos(src[q]) * N + c], 0.0), 1.0);
        r = roh * (1.0 - F);
      }
      d[(int64_t)src[q] * N + c] += r;
      kag[q] = -f.aging_gain * r;
    }
  }
  if (ksrc) {
    ksrc[c] = k0;
    ksrc[N + c] = k1;
    for (int q = 0; q < 4; ++q) ksrc[(int64_t)(2 + q) * N + c] = kag[q];
  }
}

struct CouplingSrc {
  const double* c[8];
  int shift[8];
};

// e and out may alias: each (bin, cell) is read and written by one thread.
__global__ void k_source_coupling(int64_t N, int n_src, CouplingSrc S, const double* __restrict__ kdiag,
                                  const double* e, double* out) {
  const int tau = blockIdx.y;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (int64_t)gridDim.x * blockDim.x) {
    double v = e[(int64_t)tau * N + p];
    for (int q = 0; q < n_src; ++q)
      v -= kdiag[((int64_t)q * 8 + tau) * N + p] * S.c[q][(int64_t)(tau + S.shift[q]) * N + p];
    out[(int64_t)tau * N + p] = v;
  }
}

// Archive-driven NOx -> TotalNO3 rate, one thread per cell
// (nox_to_no3_rate.py:94-155; oxidants.py:142-206 for the JPL rate, the N2O5
// equilibrium constant, the air number density and the N2O5 mean speed).
constexpr double kAvogadro = 6.02214076e23;
constexpr double kBoltzmann = 1.380649e-23;
constexpr double kRGas = 8.31446;
constexpr double kPi = 3.14159265358979323846;
// element-to-compound mass ratios (orbit/core/constants.py:9-15)
constexpr double kSToSO4 = 96.0632 / 32.0655;
constexpr double kNToNH4 = 18.03851 / 14.0067;
constexpr double kNToNO3 = 62.00501 / 14.0067;

__global__ void k_nox_rate(int64_t N, orbit_oxidant_fields_t f, int night, double* __restrict__ rate) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const double T = f.temperature[c], P = f.pressure[c];
  const double M = P * kAvogadro / (kRGas * T) * 1e-6;  // molec/cm3
  const double no = f.no ? f.no[c] * 1e-9 * M : 0.0;
  const double no2 = f.no2[c] * 1e-9 * M;
  const double nox = no + no2;
  const double safe = nox > 0.0 ? nox : 1.0;
  const double f_no2 = nox > 0.0 ? no2 / safe : 1.0;
  // OH + NO2 (+M): JPL Troe form, k0 = 1.8e-30 (T/298)^-3 M, kinf = 2.8e-11, Fc = 0.6
  const double k0 = 1.8e-30 * pow(T / 298.0, -3.0) * M;
  const double ratio = k0 / 2.8e-11;
  const double lg = log10(ratio);
  const double k_oh = (k0 / (1.0 + ratio)) * pow(0.6, 1.0 / (1.0 + lg * lg));
  const double k_day = k_oh * f.oh[c] * f_no2;
  double k_night = 0.0;
  if (night && f.no3rad) {
    const double no3 = f.no3rad[c] * 1e-9 * M;
    const double n2o5 = 5.8e-27 * exp(10840.0 / T) * no2 * no3;
    double fine = 0.0;  // ug/m3 of compound mass
    if (f.p_s) fine = fine + f.p_s[c] * kSToSO4;
    if (f.p_nh) fine = fine + f.p_nh[c] * kNToNH4;
    if (f.p_no) fine = fine + f.p_no[c] * kNToNO3;
    if (f.dust_fine) fine = fine + f.dust_fine[c];
    if (f.sea_salt_fine) fine = fine + f.sea_salt_fine[c];
    const double area = fine * 1e-9 * (3.0 / (1700.0 * 0.15e-6)) * 1e-2;  // cm2/cm3
    const double v = sqrt(8.0 * kBoltzmann * T / (kPi * (108.01e-3 / kAvogadro))) * 100.0;  // cm/s
    const double k_het = 0.25 * 0.02 * v * area;
    k_night = nox > 0.0 ? 2.0 * k_het * n2o5 / safe : 0.0;
  }
  rate[c] = k_day + k_night;
}

}  // namespace
}  // namespace orbit

extern "C" {

int orbit_nox_to_no3_rate(int64_t n_cells, const orbit_oxidant_fields_t* f, int disable_night, double* rate,
                          orbit_stream_t stream) {
  using namespace orbit;
  if (!f || !rate || n_cells < 1 || !f->temperature || !f->pressure || !f->oh || !f->no2) {
    set_last_error("orbit_nox_to_no3_rate: missing argument or required field (T, P, OH, NO2)");
    return ORBIT_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  k_nox_rate<<<(unsigned)((n_cells + 127) / 128), 128, 0, st>>>(n_cells, *f, disable_night ? 0 : 1, rate);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

int orbit_species_diagonals(int nz, int ny, int nx, const orbit_species_fields_t* f, double* d, double* k_src,
                            orbit_stream_t stream) {
  using namespace orbit;
  if (!f || !d || nz < 1 || ny < 1 || nx < 1 || !f->Dz || !f->particle_dry_dep || !f->nh3_dry_dep ||
      !f->so2_dry_dep || !f->nox_dry_dep || !f->particle_wet_dep || !f->other_gas_wet_dep || !f->so2_wet_dep ||
      !f->nh_part) {
    set_last_error("orbit_species_diagonals: missing argument or required field");
    return ORBIT_ERR_ARG;
  }
  const int64_t N = (int64_t)nz * ny * nx;
  cudaStream_t st = (cudaStream_t)stream;
  k_species_diag<<<(unsigned)((N + 127) / 128), 128, 0, st>>>(nz, ny, nx, *f, d, k_src);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

int orbit_source_coupling(int64_t N, int n_src, const double* const* c_src, const int* shift, const double* kdiag,
                          const double* e, double* out, orbit_stream_t stream) {
  using namespace orbit;
  if (N < 1 || n_src < 0 || n_src > 8 || !e || !out || (n_src > 0 && (!c_src || !shift || !kdiag))) {
    set_last_error("orbit_source_coupling: bad arguments (at most 8 sources)");
    return ORBIT_ERR_ARG;
  }
  CouplingSrc S{};
  for (int q = 0; q < n_src; ++q) {
    if (!c_src[q] || shift[q] < 0 || shift[q] > 1) {
      set_last_error("orbit_source_coupling: null source orbit or shift not 0/1");
      return ORBIT_ERR_ARG;
    }
    S.c[q] = c_src[q];
    S.shift[q] = shift[q];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t bx = std::min<int64_t>((N + 255) / 256, 4096);
  k_source_coupling<<<dim3((unsigned)bx, 8), 256, 0, st>>>(N, n_src, S, kdiag, e, out);
  note_launch();
  ORBIT_CUDA_TRY(cudaGetLastError());
  return ORBIT_OK;
}

}  // extern "C"
