// Flow files: SAVE_FLOW / READ_FLOW (for/diablo_io.f:201-404) and the
// physical-space fields of the HDF5 flow files (for/hdf5.f:5-544).
//
// Unformatted path.  The reference's flow files without ".h5" are Fortran
// unformatted sequential files: a header record (NX, NY, NZ, NUM_PER_DIR as
// INTEGER*4, TIME as REAL*8, TIME_STEP as INTEGER*4) and one data record of
// retained modes, each record framed by 4-byte little-endian length markers
// (gfortran's convention).  The data record lists (((CU(I,K,J), I=0..NKX),
// K=0..TNKZ), J=...) -- kx fastest, then packed kz, then y -- which is this
// library's compact layout, so a record is a run of contiguous planes:
//   channel  CU1 J=1..NY, CU2 J=2..NY, CU3 J=1..NY; scalar files J=0..NY on
//            write but J=1..NY on read (for/diablo_io.f:379 vs :279): a file
//            SAVE_FLOW wrote comes back one plane lower, and that is kept
//   periodic CU1..CU3 and CTH over all ky planes J=0..TNKY
//
// HDF5 path.  The datasets of /Timestep are physical fields on planes
// 1..NY stored as Fortran tmp(NX,NY,NZ) (for/hdf5.f:1242-1281), i.e. C order
// [NZ][NY][NX]; V is first moved onto GYF by G2GF and brought back by GF2G on
// read (for/hdf5.f:1176-1238).  This file produces and consumes those
// arrays; the host writes and reads the HDF5 file with its own library.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "dg_internal.cuh"

namespace {

constexpr size_t kMaxRecord = 2147483647;  // one gfortran record marker

bool put_marker(FILE *f, size_t n) {
  const int32_t m = (int32_t)n;
  return fwrite(&m, 4, 1, f) == 1;
}

int write_header(FILE *f, const dg_handle *h, int time_step, double time) {
  const int32_t dims[4] = {h->NX, h->NY, h->NZ, h->p.num_per_dir};
  const int32_t ts = time_step;
  if (!put_marker(f, 28) || fwrite(dims, 4, 4, f) != 4 || fwrite(&time, 8, 1, f) != 1 ||
      fwrite(&ts, 4, 1, f) != 1 || !put_marker(f, 28))
    return DG_ERR_ARG;
  return DG_OK;
}

// one record holding planes [j0, j1] of each listed spectral field
int write_record(FILE *f, dg_handle *h, const std::vector<const double2 *> &src,
                 const std::vector<int> &j0, const std::vector<int> &j1) {
  size_t tot = 0;
  for (size_t q = 0; q < src.size(); q++) tot += sizeof(double2) * h->ss * (j1[q] - j0[q] + 1);
  if (tot > kMaxRecord) {
    dg_set_error("flow record above 2 GiB (gfortran subrecords are not written)");
    return DG_ERR_DIMS;
  }
  if (!put_marker(f, tot)) return DG_ERR_ARG;
  std::vector<double2> buf;
  for (size_t q = 0; q < src.size(); q++) {
    const size_t n = (size_t)h->ss * (j1[q] - j0[q] + 1);
    buf.resize(n);
    DG_CUDA(cudaMemcpyAsync(buf.data(), src[q] + (long)j0[q] * h->ss, n * sizeof(double2),
                            cudaMemcpyDeviceToHost, h->st));
    DG_CUDA(cudaStreamSynchronize(h->st));
    if (fwrite(buf.data(), sizeof(double2), n, f) != n) return DG_ERR_ARG;
  }
  if (!put_marker(f, tot)) return DG_ERR_ARG;
  return DG_OK;
}

struct Reader {
  FILE *f = nullptr;
  std::vector<unsigned char> rec;
  ~Reader() {
    if (f) fclose(f);
  }
  // next record into rec
  bool next() {
    int32_t m = 0, t = 0;
    if (fread(&m, 4, 1, f) != 1 || m < 0) return false;
    rec.resize((size_t)m);
    if (m > 0 && fread(rec.data(), 1, (size_t)m, f) != (size_t)m) return false;
    return fread(&t, 4, 1, f) == 1 && t == m;
  }
};

int read_header(Reader &r, const dg_handle *h, double *time, int *time_step, const char *fname) {
  if (!r.next() || r.rec.size() < 28) {
    dg_set_error((std::string("not a flow file header: ") + fname).c_str());
    return DG_ERR_ARG;
  }
  int32_t dims[4], ts;
  memcpy(dims, r.rec.data(), 16);
  memcpy(time, r.rec.data() + 16, 8);
  memcpy(&ts, r.rec.data() + 24, 4);
  *time_step = ts;
  // for/diablo_io.f:245-248
  if (dims[0] != h->NX || dims[1] != h->NY || dims[2] != h->NZ) {
    dg_set_error("Error: old flowfield wrong dimensions.");
    return DG_ERR_DIMS;
  }
  if (dims[3] != h->p.num_per_dir) {
    dg_set_error("Error: old flowfield wrong NUM_PER_DIR.");
    return DG_ERR_DIMS;
  }
  return DG_OK;
}

// planes [j0, j1] of each field from the current record, in order; the
// record may hold more (a Fortran READ takes a prefix of its record)
int scatter_record(Reader &r, dg_handle *h, const std::vector<double2 *> &dst,
                   const std::vector<int> &j0, const std::vector<int> &j1) {
  size_t need = 0;
  for (size_t q = 0; q < dst.size(); q++) need += sizeof(double2) * h->ss * (j1[q] - j0[q] + 1);
  if (r.rec.size() < need) {
    dg_set_error("flow record shorter than the fields it must hold");
    return DG_ERR_DIMS;
  }
  size_t off = 0;
  for (size_t q = 0; q < dst.size(); q++) {
    const size_t n = sizeof(double2) * h->ss * (j1[q] - j0[q] + 1);
    DG_CUDA(cudaMemcpyAsync(dst[q] + (long)j0[q] * h->ss, r.rec.data() + off, n,
                            cudaMemcpyHostToDevice, h->st));
    off += n;
  }
  DG_CUDA(cudaStreamSynchronize(h->st));
  return DG_OK;
}

}  // namespace

extern "C" int diablo_save_flow(dg_handle *h, int time_step, const char *fname,
                                const char *const *fname_th) {
  if (!h || !fname) return DG_ERR_ARG;
  double time = 0.0, dt = 0.0;
  DG_TRY(diablo_get_time(h, &time, &dt));
  const int NY = h->NY, top = h->nplanes - 1;
  {
    FILE *f = fopen(fname, "wb");
    if (!f) {
      dg_set_error((std::string("cannot open ") + fname).c_str());
      return DG_ERR_ARG;
    }
    int s = write_header(f, h, time_step, time);
    if (s == DG_OK) {
      if (h->periodic)
        s = write_record(f, h, {h->cu[0], h->cu[1], h->cu[2]}, {0, 0, 0}, {top, top, top});
      else
        s = write_record(f, h, {h->cu[0], h->cu[1], h->cu[2]}, {1, 2, 1}, {NY, NY, NY});
    }
    if (fclose(f) != 0 && s == DG_OK) s = DG_ERR_ARG;
    DG_TRY(s);
  }
  for (int n = 0; n < h->NTH && fname_th; n++) {
    if (!fname_th[n]) continue;
    FILE *f = fopen(fname_th[n], "wb");
    if (!f) {
      dg_set_error((std::string("cannot open ") + fname_th[n]).c_str());
      return DG_ERR_ARG;
    }
    int s = write_header(f, h, time_step, time);
    // for/diablo_io.f:379 writes J=0..NY
    if (s == DG_OK) s = write_record(f, h, {h->cu[3 + n]}, {0}, {h->periodic ? top : NY});
    if (fclose(f) != 0 && s == DG_OK) s = DG_ERR_ARG;
    DG_TRY(s);
  }
  return DG_OK;
}

extern "C" int diablo_read_flow(dg_handle *h, const char *fname, const char *const *fname_th,
                                int *time_step) {
  if (!h || !fname) return DG_ERR_ARG;
  const int NY = h->NY, top = h->nplanes - 1;
  double time = 0.0, dt0 = 0.0, dt = 0.0;
  int ts = 0;
  DG_TRY(diablo_get_time(h, &dt0, &dt));
  {
    Reader r;
    r.f = fopen(fname, "rb");
    if (!r.f) {
      dg_set_error((std::string("cannot open ") + fname).c_str());
      return DG_ERR_ARG;
    }
    DG_TRY(read_header(r, h, &time, &ts, fname));
    if (!r.next()) {
      dg_set_error((std::string("truncated flow file: ") + fname).c_str());
      return DG_ERR_ARG;
    }
    // rows outside the record keep the values they had; a fresh handle holds zeros
    if (h->periodic)
      DG_TRY(scatter_record(r, h, {h->cu[0], h->cu[1], h->cu[2]}, {0, 0, 0}, {top, top, top}));
    else
      DG_TRY(scatter_record(r, h, {h->cu[0], h->cu[1], h->cu[2]}, {1, 2, 1}, {NY, NY, NY}));
  }
  for (int n = 0; n < h->NTH && fname_th; n++) {
    if (!fname_th[n]) continue;
    Reader r;
    r.f = fopen(fname_th[n], "rb");
    if (!r.f) {
      dg_set_error((std::string("cannot open ") + fname_th[n]).c_str());
      return DG_ERR_ARG;
    }
    int t2 = 0;
    DG_TRY(read_header(r, h, &time, &t2, fname_th[n]));  // TIME, TIME_STEP as the reference
    ts = t2;
    if (!r.next()) {
      dg_set_error((std::string("truncated flow file: ") + fname_th[n]).c_str());
      return DG_ERR_ARG;
    }
    // for/diablo_io.f:279 reads J=1..NY (periodic: J=0..TNKY)
    if (h->periodic) DG_TRY(scatter_record(r, h, {h->cu[3 + n]}, {0}, {top}));
    else DG_TRY(scatter_record(r, h, {h->cu[3 + n]}, {1}, {NY}));
  }
  DG_TRY(diablo_set_time(h, time, dt));
  if (time_step) *time_step = ts;
  // initial boundary conditions (for/diablo_io.f:296-301); channel only: on a
  // periodic state these routines would overwrite the ky = 0 and 1 planes
  if (!h->periodic) DG_TRY(diablo_apply_bc_vel(h));
  return DG_OK;
}

// ------------------------------------------------------------ HDF5 fields

namespace {

// physical field in the reference layout (0:NX+1, 0:NZ+1, 0:NY+1) from a spectral field
int to_phys_ref(dg_handle *h, int field, std::vector<double> &spec, std::vector<double> &phys) {
  const long pplane = (long)(h->NX + 2) * (h->NZ + 2);
  spec.assign((size_t)pplane * (h->NY + 2), 0.0);
  phys.assign((size_t)pplane * (h->NY + 2), 0.0);
  DG_TRY(diablo_get_field(h, field, spec.data(), DG_LAYOUT_REFERENCE, DG_HOST));
  return diablo_fft_xz_to_physical(h, spec.data(), phys.data(), 0, h->NY + 1, DG_HOST);
}

int from_phys_ref(dg_handle *h, int field, std::vector<double> &phys, std::vector<double> &spec) {
  const long pplane = (long)(h->NX + 2) * (h->NZ + 2);
  spec.assign((size_t)pplane * (h->NY + 2), 0.0);
  DG_TRY(diablo_fft_xz_to_fourier(h, phys.data(), spec.data(), 0, h->NY + 1, DG_HOST));
  return diablo_set_field(h, field, spec.data(), DG_LAYOUT_REFERENCE, DG_HOST);
}

}  // namespace

extern "C" int diablo_flow_fields_physical(dg_handle *h, double *U, double *V, double *W,
                                           double *TH, double *P) {
  if (!h || h->periodic) return DG_ERR_ARG;
  const int NX = h->NX, NY = h->NY, NZ = h->NZ;
  const long rx = NX + 2, pplane = rx * (NZ + 2);
  std::vector<double> spec, phys;
  // SWAPZY (for/hdf5.f:1242-1259): out(x+1, y, z+1) = in(x, z, y), y = 1..NY
  auto swap_out = [&](double *out) {
    for (int z = 0; z < NZ; z++)
      for (int y = 1; y <= NY; y++)
        for (int x = 0; x < NX; x++)
          out[((long)z * NY + (y - 1)) * NX + x] = phys[(size_t)y * pplane + (long)z * rx + x];
  };
  auto one = [&](int field, double *out, bool g2gf) -> int {
    if (!out) return DG_OK;
    DG_TRY(to_phys_ref(h, field, spec, phys));
    if (g2gf) {
      // G2GF (for/hdf5.f:1176-1193): onto GYF with the wall values copied in
      for (int z = 0; z < NZ; z++)
        for (int x = 0; x < NX; x++) {
          double *v = phys.data() + (long)z * rx + x;
          v[1 * pplane] = v[2 * pplane];
          v[(long)(NY + 1) * pplane] = v[(long)NY * pplane];
          for (int y = 1; y <= NY; y++)
            v[(long)y * pplane] = 0.5 * (v[(long)y * pplane] + v[(long)(y + 1) * pplane]);
        }
    }
    swap_out(out);
    return DG_OK;
  };
  DG_TRY(one(DG_CU1, U, false));
  DG_TRY(one(DG_CU2, V, true));
  DG_TRY(one(DG_CU3, W, false));
  for (int n = 0; n < h->NTH && TH; n++) DG_TRY(one(DG_CTH + n, TH + (long)n * NZ * NY * NX, false));
  DG_TRY(one(DG_CP, P, false));
  return DG_OK;
}

extern "C" int diablo_flow_fields_from_physical(dg_handle *h, const double *U, const double *V,
                                                const double *W, const double *TH, const double *P,
                                                double time) {
  if (!h || h->periodic || !U || !V || !W || (h->NTH > 0 && !TH)) return DG_ERR_ARG;
  const int NX = h->NX, NY = h->NY, NZ = h->NZ;
  const long rx = NX + 2, pplane = rx * (NZ + 2);
  std::vector<double> spec, phys;
  // SWAPYZ (for/hdf5.f:1264-1281): zero, then in(x, z, y) = tmp(x+1, y, z+1), y = 1..NY
  auto swap_in = [&](const double *in) {
    phys.assign((size_t)pplane * (NY + 2), 0.0);
    for (int z = 0; z < NZ; z++)
      for (int y = 1; y <= NY; y++)
        for (int x = 0; x < NX; x++)
          phys[(size_t)y * pplane + (long)z * rx + x] = in[((long)z * NY + (y - 1)) * NX + x];
  };
  swap_in(U);
  DG_TRY(from_phys_ref(h, DG_CU1, phys, spec));
  swap_in(V);
  // GF2G (for/hdf5.f:1197-1238): back onto GY, then the zero-mass-flux walls
  for (int z = 0; z < NZ; z++)
    for (int x = 0; x < NX; x++) {
      double *v = phys.data() + (long)z * rx + x;
      v[(long)(NY + 1) * pplane] = v[(long)NY * pplane];
      for (int y = NY; y >= 1; y--)
        v[(long)y * pplane] = 2 * v[(long)y * pplane] - v[(long)(y + 1) * pplane];
      v[1 * pplane] = -v[2 * pplane];
      v[(long)(NY + 1) * pplane] = -v[(long)NY * pplane];
    }
  DG_TRY(from_phys_ref(h, DG_CU2, phys, spec));
  swap_in(W);
  DG_TRY(from_phys_ref(h, DG_CU3, phys, spec));
  for (int n = 0; n < h->NTH; n++) {
    swap_in(TH + (long)n * NZ * NY * NX);
    DG_TRY(from_phys_ref(h, DG_CTH + n, phys, spec));
  }
  double t0 = 0.0, dt = 0.0;
  DG_TRY(diablo_get_time(h, &t0, &dt));
  DG_TRY(diablo_set_time(h, time, dt));
  if (P) {
    swap_in(P);
    DG_TRY(from_phys_ref(h, DG_CP, phys, spec));
  }
  // for/hdf5.f:509-511 (COURANT with VARIABLE_DT) and :530-538 (POISSON_P_CHAN
  // when the file holds no pressure)
  if (h->p.variable_dt) DG_TRY(diablo_courant(h));
  if (!P) DG_TRY(diablo_poisson_p_chan(h));
  return DG_OK;
}
