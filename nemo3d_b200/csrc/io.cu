// Result files in the reference's <HDR> format, so that its post-processing
// tools read GPU results: a text header (writeHeader,
// nemo3d/src/io/fileformat.c:182-204) followed by native-endian binary
// records.  Eigenvalues: the nd_Ek file of writeEigenvalues
// (nemo3d/src/io/i_3dout_files.c:1886-1975), records {kx, ky, kz, E};
// eigenvectors: the nd_evec files of writeEigenvector (i_3dout_files.c:
// 1342-1357, header of writeHeader_siteInfo "basis", i_3dout_files.c:116-200),
// records {wf.r, wf.i} for every basis state.  Host code only.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tbgpu_internal.cuh"

namespace tbgpu {
namespace {

// "<HDR>", record format, record dimensions, user data, "<\HDR>"
bool write_header(FILE *fp, const char *fmt, const std::vector<int> &dim,
                  const std::vector<std::string> &lbl, const std::vector<std::string> &usr) {
  if (std::fprintf(fp, "<HDR>\n%-20s = %s\n", "record format", fmt) < 0) return false;
  for (size_t i = 0; i < dim.size(); i++) {
    const std::string key = "record dimension " + std::to_string(i + 1);
    std::fprintf(fp, "%-20s = %-10d %s\n", key.c_str(), dim[i], lbl[i].c_str());
  }
  for (size_t i = 0; i < usr.size(); i++) {
    const std::string key = "user data " + std::to_string(i + 1);
    std::fprintf(fp, "%-20s =%s\n", key.c_str(), usr[i].c_str());
  }
  return std::fprintf(fp, "<\\HDR>") >= 0;
}

// the count of the first record dimension and the records after "<\HDR>"
bool read_ek(const char *path, int &count, std::vector<double> &data) {
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return false;
  std::string all;
  char buf[65536];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), fp)) > 0) all.append(buf, got);
  std::fclose(fp);
  const size_t end = all.find("<\\HDR>");
  const size_t dimkey = all.find("record dimension 1");
  if (end == std::string::npos || dimkey == std::string::npos || dimkey > end) return false;
  const size_t eq = all.find('=', dimkey);
  if (eq == std::string::npos || eq > end) return false;
  count = std::atoi(all.c_str() + eq + 1);
  const size_t off = end + 6;
  if (count < 0 || all.size() < off + sizeof(double) * 4 * size_t(count)) return false;
  data.resize(size_t(count) * 4);
  std::memcpy(data.data(), all.data() + off, sizeof(double) * data.size());
  return true;
}

}  // namespace
}  // namespace tbgpu

using namespace tbgpu;

extern "C" int tbgpu_write_eigenvalues(const char *path, char mode, const double *k, int n,
                                       const double *E) {
  if (!path || (mode != 'i' && mode != 'a') || (mode == 'a' && (n < 0 || (n > 0 && !E))))
    return set_error(TBGPU_E_ARG);
  if (mode == 'i') {  // create or empty the file
    FILE *fp = std::fopen(path, "w");
    if (!fp) return set_error(TBGPU_E_ARG);
    std::fclose(fp);
    return TBGPU_OK;
  }
  // 'a': keep the records already there, rewrite the header with the new
  // count, append the new records (as writeEigenvalues does)
  int count = 0;
  std::vector<double> old;
  FILE *probe = std::fopen(path, "rb");
  const bool has = probe && std::fgetc(probe) != EOF;
  if (probe) std::fclose(probe);
  if (has && !read_ek(path, count, old)) return set_error(TBGPU_E_ARG);
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return set_error(TBGPU_E_ARG);
  const double kk[3] = {k ? k[0] : 0.0, k ? k[1] : 0.0, k ? k[2] : 0.0};
  bool ok = write_header(fp, "{real kx, real ky, real kz, real E}", {count + n},
                         {"# number of eigenvalues"},
                         {"                                        # not used"});
  if (count > 0) ok = ok && std::fwrite(old.data(), sizeof(double), old.size(), fp) == old.size();
  for (int j = 0; j < n && ok; j++) {
    const double rec[4] = {kk[0], kk[1], kk[2], E[j]};
    ok = std::fwrite(rec, sizeof(double), 4, fp) == 4;
  }
  std::fclose(fp);
  return ok ? TBGPU_OK : set_error(TBGPU_E_ARG);
}

extern "C" int tbgpu_write_eigenvector(const tbgpu_ctx *ctx, const char *path,
                                       const tbgpu_dcomplex *wf, int crystal_structure) {
  if (!ctx || !path || !wf) return set_error(TBGPU_E_ARG);
  const Ctx &c = *reinterpret_cast<const Ctx *>(ctx);
  if (!c.built) return set_error(TBGPU_E_STATE);
  const char *model = "";
  switch (c.band_model) {
    case TBGPU_SP3D5S_SO: model = "Bands_20_sp3d5ss_spin # band_model"; break;
    case TBGPU_SP3S_SO: model = "Bands_10_sp3ss_spin  # band_model"; break;
    case TBGPU_SP3D5S: model = "Bands_10_sp3d5ss_nospin  # band_model"; break;
    default: model = "Bands_5_sp3ss_nospin  # band_model"; break;  // no reference counterpart
  }
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return set_error(TBGPU_E_ARG);
  const std::string cs = std::to_string(crystal_structure) + " # crystal structure";
  bool ok = write_header(fp, "{real wf.r, real wf.i}", {c.nb, int(c.natoms)},
                         {"# order of orbital basis", "# number of atoms"}, {model, cs});
  const size_t n = size_t(c.natoms) * c.nb;
  ok = ok && std::fwrite(wf, sizeof(tbgpu_dcomplex), n, fp) == n;
  std::fclose(fp);
  return ok ? TBGPU_OK : set_error(TBGPU_E_ARG);
}

// The tridiagonal matrix and eigenvalue files of eigensolve_lanczos's saved
// state (eigen/src/lanczos.c:1692-1809): native-endian binary,
//   T:       int iterations, int processors, double t[2*iterations] with
//            t[2i] = alpha_i and t[2i-1] = beta_{i-1} (the last slot unused);
//   values:  int n, double value[n].
// On reading, the reference keeps iterations - 200 of the stored matrix
// (restoreTridiagonalMatrix, lanczos.c:1765); so does this reader.
extern "C" int tbgpu_write_tridiagonal_file(const char *path, const double *alpha,
                                            const double *beta, int iterations,
                                            int processors) {
  if (!path || !alpha || !beta || iterations < 1) return set_error(TBGPU_E_ARG);
  std::vector<double> t(2 * size_t(iterations), 0.0);
  for (int i = 0; i < iterations; i++) t[2 * size_t(i)] = alpha[i];
  for (int i = 1; i < iterations; i++) t[2 * size_t(i) - 1] = beta[i - 1];
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return set_error(TBGPU_E_ARG);
  const bool ok = std::fwrite(&iterations, sizeof(int), 1, fp) == 1 &&
                  std::fwrite(&processors, sizeof(int), 1, fp) == 1 &&
                  std::fwrite(t.data(), sizeof(double), t.size(), fp) == t.size();
  return (std::fclose(fp) == 0 && ok) ? TBGPU_OK : set_error(TBGPU_E_ARG);
}

extern "C" int tbgpu_read_tridiagonal_file(const char *path, int cap, double *alpha,
                                           double *beta, int *processors) {
  if (!path || cap < 0 || (cap > 0 && (!alpha || !beta))) return set_error(TBGPU_E_ARG);
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return set_error(TBGPU_E_ARG);
  int stored = 0, procs = 0;
  bool ok = std::fread(&stored, sizeof(int), 1, fp) == 1 &&
            std::fread(&procs, sizeof(int), 1, fp) == 1 && stored > 200;
  const int its = stored - 200;
  std::vector<double> t;
  if (ok) {
    t.resize(2 * size_t(its));
    ok = std::fread(t.data(), sizeof(double), t.size(), fp) == t.size();
  }
  std::fclose(fp);
  if (!ok) return set_error(TBGPU_E_ARG);
  if (processors) *processors = procs;
  for (int i = 0; i < its && i < cap; i++) {
    alpha[i] = t[2 * size_t(i)];
    beta[i] = i + 1 < its ? t[2 * size_t(i) + 1] : 0.0;
  }
  return its;
}

extern "C" int tbgpu_write_eigenvalue_file(const char *path, const double *values, int n) {
  if (!path || n < 0 || (n > 0 && !values)) return set_error(TBGPU_E_ARG);
  FILE *fp = std::fopen(path, "wb");
  if (!fp) return set_error(TBGPU_E_ARG);
  const bool ok = std::fwrite(&n, sizeof(int), 1, fp) == 1 &&
                  std::fwrite(values, sizeof(double), size_t(n), fp) == size_t(n);
  return (std::fclose(fp) == 0 && ok) ? TBGPU_OK : set_error(TBGPU_E_ARG);
}

extern "C" int tbgpu_read_eigenvalue_file(const char *path, int cap, double *values) {
  if (!path || cap < 0 || (cap > 0 && !values)) return set_error(TBGPU_E_ARG);
  FILE *fp = std::fopen(path, "rb");
  if (!fp) return set_error(TBGPU_E_ARG);
  int n = 0;
  bool ok = std::fread(&n, sizeof(int), 1, fp) == 1 && n >= 0;
  std::vector<double> v(ok ? size_t(n) : 0);
  if (ok) ok = std::fread(v.data(), sizeof(double), v.size(), fp) == v.size();
  std::fclose(fp);
  if (!ok) return set_error(TBGPU_E_ARG);
  for (int i = 0; i < n && i < cap; i++) values[i] = v[i];
  return n;
}
