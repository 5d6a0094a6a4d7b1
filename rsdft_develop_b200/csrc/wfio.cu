// Wavefunction checkpoint files in the reference's format.
//
// Reference: write_wf_simple (src/io_write_wf_simple_module.f90:21-276) and read_wf_simple
// (src/io_read_wf_simple_module.f90), called by write_data / read_data (src/io_module.f90:59-491)
// for the restart keywords OC / IC.  The file is a Fortran sequential unformatted file (every
// record framed by its byte length as a 4-byte integer before and after the payload), written
// by one process (IO_ctrl = 0), new layout (OC < 10):
//
//   -1 | ML, ML1, ML2, ML3 | MB, MBwr1, MBwr2 | MK, MS, MMBZ | IO_ctrl, OC, TYPE_WF |
//   LL2(3, ML) | occ(MB, MK, MS) | aa(3,3), bb(3,3), kbb(3, MK) | np(0:7) |
//   grid id, ir | band id, ir | bz id, ir | spin id, ir |
//   then one record per band, s outermost, then k, then n = MBwr1..MBwr2:
//   unk(1:ML, n, k, s) as real(8) / complex(8) (OC 1, 3) or real(4) / complex(4) (OC 4, 5).
//
// TYPE_WF is 1 for real8 and 0 for complex16 wavefunctions (as the writer sets it); the reader
// also takes 3 / 2 for single-precision records, and OC 4 / 5 mark single precision either way.
// LL2(:, i) are the grid coordinates (0-based) of the i-th point of every band record; this
// library writes its own layout (x fastest, as unk(ML0, :) is ordered), and the reader places
// each point of a file written with another layout by its LL2 entry.  The old layout (no leading
// -1: ML.. | MB.. | LL2 | occ, then the bands) is read too.  Bands beyond a k-point's active
// band count (uneven counts) are written as zeros and skipped on reading.
#include <cstdio>
#include <cstring>
#include <vector>

#include "ctx.cuh"

namespace rsdft {
namespace {

struct FFile {
  FILE* f = nullptr;
  ~FFile() {
    if (f) fclose(f);
  }
};

int put_record(FILE* f, const void* data, size_t bytes) {
  RS_CHECK(bytes < 0x7fffffffULL, RSDFT_ERR_UNSUPPORTED, "record of %zu bytes exceeds the 4-byte record marker", bytes);
  const int32_t m = (int32_t)bytes;
  RS_CHECK(fwrite(&m, 4, 1, f) == 1 && (bytes == 0 || fwrite(data, 1, bytes, f) == bytes) && fwrite(&m, 4, 1, f) == 1,
           RSDFT_ERR_IO, "write error");
  return 0;
}

template <typename T>
int put_vec(FILE* f, const std::vector<T>& v) {
  return put_record(f, v.data(), v.size() * sizeof(T));
}

// reads the next record; out receives its payload
int get_record(FILE* f, std::vector<unsigned char>& out) {
  int32_t m0 = 0, m1 = 0;
  RS_CHECK(fread(&m0, 4, 1, f) == 1, RSDFT_ERR_IO, "unexpected end of file");
  RS_CHECK(m0 >= 0, RSDFT_ERR_IO, "bad record marker %d", m0);
  out.resize((size_t)m0);
  RS_CHECK(m0 == 0 || fread(out.data(), 1, (size_t)m0, f) == (size_t)m0, RSDFT_ERR_IO, "truncated record");
  RS_CHECK(fread(&m1, 4, 1, f) == 1 && m1 == m0, RSDFT_ERR_IO, "record markers do not match (%d, %d)", m0, m1);
  return 0;
}

template <typename T>
int get_ints(FILE* f, T* v, int n, const char* what) {
  std::vector<unsigned char> r;
  RS_TRY(get_record(f, r));
  RS_CHECK(r.size() >= sizeof(T) * (size_t)n, RSDFT_ERR_IO, "record %s too short (%zu bytes)", what, r.size());
  std::memcpy(v, r.data(), sizeof(T) * (size_t)n);
  return 0;
}

int max_nband(const Ctx& c) {
  int mb = 0;
  for (int k = 0; k < c.p.nk; ++k) mb = std::max(mb, c.kp[k].nband);
  return mb;
}

}  // namespace
}  // namespace rsdft

using namespace rsdft;

extern "C" int rsdft_gpu_write_wf(const char* path, int oc, const double* occ, const double* aa, const double* bb,
                                  const double* kbb) {
  Ctx* cp = ctx();
  RS_CHECK(cp != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called");
  Ctx& c = *cp;
  RS_CHECK(path != nullptr, RSDFT_ERR_ARG, "no file name");
  RS_CHECK(oc == 1 || oc == 3 || oc == 4 || oc == 5, RSDFT_ERR_ARG, "OC must be 1, 3, 4 or 5 (got %d)", oc);
  const int ML = (int)c.ng, mk = c.p.nk, ms = c.p.nspin, mb = max_nband(c);
  for (int k = 0; k < mk; ++k)
    for (int s = 0; s < ms; ++s)
      RS_CHECK(c.kp[k].nband == 0 || c.wfn(k, s).valid, RSDFT_ERR_STATE,
               "no wavefunctions resident for (k,s)=(%d,%d)", k + 1, s + 1);
  const bool sp = oc == 4 || oc == 5;
  const int nc = c.cplx ? 2 : 1;
  FFile ff;
  ff.f = fopen(path, "wb");
  RS_CHECK(ff.f != nullptr, RSDFT_ERR_IO, "cannot open %s for writing", path);
  FILE* f = ff.f;
  RS_TRY(put_vec<int32_t>(f, {-1}));
  RS_TRY(put_vec<int32_t>(f, {ML, c.p.n1, c.p.n2, c.p.n3}));
  RS_TRY(put_vec<int32_t>(f, {mb, 1, mb}));
  RS_TRY(put_vec<int32_t>(f, {mk, ms, mk}));
  RS_TRY(put_vec<int32_t>(f, {0, oc, c.cplx ? 0 : 1}));
  {
    std::vector<int32_t> ll((size_t)3 * ML);
    size_t i = 0;
    for (int i3 = 0; i3 < c.p.n3; ++i3)
      for (int i2 = 0; i2 < c.p.n2; ++i2)
        for (int i1 = 0; i1 < c.p.n1; ++i1, ++i) {
          ll[3 * i] = i1;
          ll[3 * i + 1] = i2;
          ll[3 * i + 2] = i3;
        }
    RS_TRY(put_vec(f, ll));
  }
  {
    std::vector<double> o((size_t)mb * mk * ms, 0.0);
    if (occ) std::memcpy(o.data(), occ, sizeof(double) * o.size());
    RS_TRY(put_vec(f, o));
  }
  {
    std::vector<double> g((size_t)18 + 3 * mk, 0.0);
    if (aa) std::memcpy(g.data(), aa, sizeof(double) * 9);
    if (bb) std::memcpy(g.data() + 9, bb, sizeof(double) * 9);
    if (kbb) std::memcpy(g.data() + 18, kbb, sizeof(double) * 3 * mk);
    RS_TRY(put_vec(f, g));
  }
  RS_TRY(put_vec<int32_t>(f, {1, 1, 1, 1, 1, 1, 1, 1}));  // np(0:7): one process
  RS_TRY(put_vec<int32_t>(f, {0, ML}));
  RS_TRY(put_vec<int32_t>(f, {0, mb}));
  RS_TRY(put_vec<int32_t>(f, {0, mk}));
  RS_TRY(put_vec<int32_t>(f, {0, ms}));
  // band records, staged one band at a time through pinned host memory
  const size_t nreal = (size_t)ML * nc;
  const size_t esz = c.mixed ? 4 : 8;
  void* stage = nullptr;
  RS_CUDA(cudaMallocHost(&stage, nreal * esz));
  std::vector<unsigned char> rec(nreal * (sp ? 4 : 8));
  int rc = 0;
  for (int s = 0; s < ms && rc == 0; ++s)
    for (int k = 0; k < mk && rc == 0; ++k)
      for (int n = 0; n < mb && rc == 0; ++n) {
        if (n < c.kp[k].nband) {
          const char* src = reinterpret_cast<const char*>(c.wfn(k, s).psi.p) + (size_t)n * nreal * esz;
          cudaError_t e = cudaMemcpyAsync(stage, src, nreal * esz, cudaMemcpyDeviceToHost, c.stream);
          if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
          if (e != cudaSuccess) {
            set_error(RSDFT_ERR_CUDA, "band copy for the wf file: %s", cudaGetErrorString(e));
            rc = RSDFT_ERR_CUDA;
            break;
          }
          if (sp && c.mixed) {
            std::memcpy(rec.data(), stage, nreal * 4);
          } else if (sp) {
            const double* d = static_cast<const double*>(stage);
            float* o = reinterpret_cast<float*>(rec.data());
            for (size_t i = 0; i < nreal; ++i) o[i] = (float)d[i];
          } else if (c.mixed) {
            const float* d = static_cast<const float*>(stage);
            double* o = reinterpret_cast<double*>(rec.data());
            for (size_t i = 0; i < nreal; ++i) o[i] = (double)d[i];
          } else {
            std::memcpy(rec.data(), stage, nreal * 8);
          }
        } else {
          std::fill(rec.begin(), rec.end(), (unsigned char)0);
        }
        rc = put_record(f, rec.data(), rec.size());
      }
  cudaFreeHost(stage);
  return rc;
}

extern "C" int rsdft_gpu_read_wf(const char* path, double* occ) {
  Ctx* cp = ctx();
  RS_CHECK(cp != nullptr, RSDFT_ERR_STATE, "rsdft_gpu_init has not been called");
  Ctx& c = *cp;
  RS_CHECK(path != nullptr, RSDFT_ERR_ARG, "no file name");
  FFile ff;
  ff.f = fopen(path, "rb");
  RS_CHECK(ff.f != nullptr, RSDFT_ERR_IO, "cannot open %s", path);
  FILE* f = ff.f;
  int32_t first = 0;
  RS_TRY(get_ints(f, &first, 1, "head"));
  int32_t g4[4], b3[3], kms[3] = {c.p.nk, c.p.nspin, c.p.nk}, ioc[3] = {0, 1, c.cplx ? 0 : 1};
  const bool newfmt = first < 0;
  if (newfmt) {
    RS_TRY(get_ints(f, g4, 4, "ML"));
  } else {
    rewind(f);
    RS_TRY(get_ints(f, g4, 4, "ML"));
  }
  RS_TRY(get_ints(f, b3, 3, "MB"));
  if (newfmt) {
    RS_TRY(get_ints(f, kms, 3, "MK"));
    RS_TRY(get_ints(f, ioc, 3, "IO_ctrl"));
  }
  const int ML = g4[0], MB = b3[0], MB1 = b3[1], MB2 = b3[2], MK = kms[0], MS = kms[1];
  const int IOc = ioc[0], OC = ioc[1], TW = ioc[2];
  RS_CHECK(ML == (int)c.ng && g4[1] == c.p.n1 && g4[2] == c.p.n2 && g4[3] == c.p.n3, RSDFT_ERR_ARG,
           "grid of the file (%d: %d %d %d) differs from the context (%zu: %d %d %d)", ML, g4[1], g4[2], g4[3], c.ng,
           c.p.n1, c.p.n2, c.p.n3);
  RS_CHECK(MK == c.p.nk && MS == c.p.nspin, RSDFT_ERR_ARG, "file holds %d k-points x %d spins, context %d x %d", MK, MS,
           c.p.nk, c.p.nspin);
  RS_CHECK(IOc == 0, RSDFT_ERR_UNSUPPORTED, "IO_ctrl %d (split files) is not read here", IOc);
  RS_CHECK(MB1 >= 1 && MB2 >= MB1 && MB2 <= MB, RSDFT_ERR_IO, "bad band range %d..%d of %d", MB1, MB2, MB);
  const bool fcplx = TW == 0 || TW == 2;
  const bool fsp = TW == 2 || TW == 3 || OC == 4 || OC == 5;
  std::vector<int32_t> ll((size_t)3 * ML);
  RS_TRY(get_ints(f, ll.data(), 3 * ML, "LL2"));
  {
    std::vector<double> o((size_t)MB * MK * MS);
    RS_TRY(get_ints(f, o.data(), (int)o.size(), "occ"));
    if (occ) std::memcpy(occ, o.data(), sizeof(double) * o.size());
  }
  if (newfmt) {
    std::vector<unsigned char> skip;
    for (int r = 0; r < 6; ++r) RS_TRY(get_record(f, skip));  // aa bb kbb | np | grid, band, bz, spin id/ir
  }
  // file point i -> grid index of this library's layout
  std::vector<size_t> to((size_t)ML);
  for (int i = 0; i < ML; ++i) {
    const int i1 = ll[3 * i], i2 = ll[3 * i + 1], i3 = ll[3 * i + 2];
    RS_CHECK(i1 >= 0 && i1 < c.p.n1 && i2 >= 0 && i2 < c.p.n2 && i3 >= 0 && i3 < c.p.n3, RSDFT_ERR_IO,
             "grid map entry %d out of range (%d %d %d)", i, i1, i2, i3);
    to[i] = ((size_t)i3 * c.p.n2 + i2) * c.p.n1 + i1;
  }
  const int nc = c.cplx ? 2 : 1;
  const size_t nreal = (size_t)ML * nc;
  const size_t esz = c.mixed ? 4 : 8;
  const size_t fes = (fsp ? 4 : 8) * (fcplx ? 2 : 1);
  for (int k = 0; k < MK; ++k)
    for (int s = 0; s < MS; ++s) {
      WaveFns& w = c.wfn(k, s);
      RS_TRY(w.psi.ensure(esz * nreal * (size_t)c.kp[k].nband));
    }
  void* stage = nullptr;
  RS_CUDA(cudaMallocHost(&stage, nreal * esz));
  std::vector<unsigned char> rec;
  std::vector<double> val(nreal);
  int rc = 0;
  for (int s = 0; s < MS && rc == 0; ++s)
    for (int k = 0; k < MK && rc == 0; ++k)
      for (int n = MB1 - 1; n < MB2 && rc == 0; ++n) {
        rc = get_record(f, rec);
        if (rc) break;
        if (rec.size() != (size_t)ML * fes) {
          set_error(RSDFT_ERR_IO, "band record of %zu bytes, expected %zu", rec.size(), (size_t)ML * fes);
          rc = RSDFT_ERR_IO;
          break;
        }
        if (n >= c.kp[k].nband) continue;
        // values in this library's layout; a complex file read into a real context keeps the
        // real part, a real file read into a complex context gets zero imaginary parts
        std::fill(val.begin(), val.end(), 0.0);
        for (int i = 0; i < ML; ++i) {
          double re, im = 0.0;
          if (fsp) {
            const float* p = reinterpret_cast<const float*>(rec.data());
            re = fcplx ? p[2 * i] : p[i];
            if (fcplx) im = p[2 * i + 1];
          } else {
            const double* p = reinterpret_cast<const double*>(rec.data());
            re = fcplx ? p[2 * i] : p[i];
            if (fcplx) im = p[2 * i + 1];
          }
          val[to[i] * nc] = re;
          if (nc == 2) val[to[i] * 2 + 1] = im;
        }
        if (c.mixed) {
          float* o = static_cast<float*>(stage);
          for (size_t i = 0; i < nreal; ++i) o[i] = (float)val[i];
        } else {
          std::memcpy(stage, val.data(), nreal * 8);
        }
        char* dst = reinterpret_cast<char*>(c.wfn(k, s).psi.p) + (size_t)n * nreal * esz;
        cudaError_t e = cudaMemcpyAsync(dst, stage, nreal * esz, cudaMemcpyHostToDevice, c.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess) {
          set_error(RSDFT_ERR_CUDA, "band copy from the wf file: %s", cudaGetErrorString(e));
          rc = RSDFT_ERR_CUDA;
        }
      }
  cudaFreeHost(stage);
  if (rc) return rc;
  for (int k = 0; k < MK; ++k)
    for (int s = 0; s < MS; ++s) c.wfn(k, s).valid = true;
  return 0;
}
