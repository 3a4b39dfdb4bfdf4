// chns_io.cu -- field files in the reference's format (write_array.c, read_array.c).
//
// Raw FP64 nx x ny arrays, row-major with x the slow index and no header: the
// layout write_array_real produces after gathering the slabs (write_array.c:18-46)
// and read_array_real consumes (read_array.c:12-40).  The real-space fields are
// computed on the device (ifft, optionally after truncation) and written by the host.
#include <cuda_runtime.h>
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <string>
#include <vector>

#include "chns_internal.h"

namespace {

int ensure_dir(const std::string& d) {
  if (mkdir(d.c_str(), 0755) == 0 || errno == EEXIST) return CHNS_OK;
  return CHNS_ERR_IO;
}

int write_raw(const std::string& path, const std::vector<double>& a) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return CHNS_ERR_IO;
  const size_t w = fwrite(a.data(), sizeof(double), a.size(), f);
  const int rc = fclose(f);
  return (w == a.size() && rc == 0) ? CHNS_OK : CHNS_ERR_IO;
}

int read_raw(const char* path, std::vector<double>& a) {
  FILE* f = fopen(path, "rb");
  if (!f) return CHNS_ERR_IO;
  const size_t r = fread(a.data(), sizeof(double), a.size(), f);
  fclose(f);
  return r == a.size() ? CHNS_OK : CHNS_ERR_IO;
}

}  // namespace

extern "C" {

int chns_write_fields(chns_ctx* c, const char* dir, int index, int truncate) {
  if (!c || !dir) return CHNS_ERR_ARG;
  const std::string base(dir);
  int rc = ensure_dir(base + "/vort");
  if (!rc && c->p.model != CHNS_MODEL_NS) rc = ensure_dir(base + "/phase_field");
  if (rc) return rc;
  const size_t nn = (size_t)c->n * c->n;
  std::vector<double> host(nn);
  const std::string idx = "." + std::to_string(index);
  const char* names[3][3] = {{"vort/wz", nullptr, nullptr},
                             {"vort/wz", "phase_field/phi", nullptr},
                             {"vort/wz", "phase_field/phi1", "phase_field/phi2"}};
  for (int f = 0; f <= c->p.model; f++) {
    rc = chns_field_to_realdbl(c, f, truncate ? 1 : 0);
    if (rc) return rc;
    if (cudaMemcpyAsync(host.data(), c->realdbl, nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess)
      return CHNS_ERR_CUDA;
    rc = write_raw(base + "/" + names[c->p.model][f] + idx, host);
    if (rc) return rc;
  }
  return CHNS_OK;
}

int chns_read_phase(chns_ctx* c, const char* path1, const char* path2) {
  if (!c || c->p.model == CHNS_MODEL_NS || !path1 || (c->p.model == CHNS_MODEL_TERNARY && !path2))
    return CHNS_ERR_ARG;
  const size_t nn = (size_t)c->n * c->n;
  std::vector<double> a(nn), b;
  int rc = read_raw(path1, a);
  if (rc) return rc;
  if (c->p.model == CHNS_MODEL_TERNARY) {
    b.resize(nn);
    rc = read_raw(path2, b);
    if (rc) return rc;
  }
  return chns_set_phase_real(c, a.data(), b.empty() ? nullptr : b.data(), CHNS_HOST);
}

// checkpoint file: magic, the chns_params the context was created with (padding
// zeroed), then the spectral fields (FFTW layout, FP64) of the model
static const char kCkptMagic[8] = {'C', 'H', 'N', 'S', 'C', 'K', 'P', '2'};

static chns_params canonical(const chns_params& a) {
  chns_params q;
  memset(&q, 0, sizeof(q));
  q.model = a.model;
  q.precision = a.precision;
  q.nx = a.nx;
  q.ny = a.ny;
  q.lx = a.lx;
  q.ly = a.ly;
  q.dt = a.dt;
  q.nu = a.nu;
  q.lambda = a.lambda;
  q.sigma = a.sigma;
  q.epsilon = a.epsilon;
  q.sigma12 = a.sigma12;
  q.sigma13 = a.sigma13;
  q.sigma23 = a.sigma23;
  q.xlambda = a.xlambda;
  q.dealias_div = a.dealias_div;
  q.coef_mode = a.coef_mode;
  q.force_amp = a.force_amp;
  q.force_k = a.force_k;
  q.filter = a.filter;
  return q;
}

int chns_save(chns_ctx* c, const char* path) {
  if (!c || !path) return CHNS_ERR_ARG;
  const size_t ncx = (size_t)c->n * c->nr;
  std::vector<double> f[3];
  for (int k = 0; k <= c->p.model; k++) f[k].resize(2 * ncx);
  int rc = chns_get_state(c, f[0].data(), c->p.model >= 1 ? f[1].data() : nullptr,
                          c->p.model == 2 ? f[2].data() : nullptr, CHNS_HOST);
  if (rc) return rc;
  FILE* fp = fopen(path, "wb");
  if (!fp) return CHNS_ERR_IO;
  const chns_params q = canonical(c->p);
  bool ok = fwrite(kCkptMagic, 1, sizeof(kCkptMagic), fp) == sizeof(kCkptMagic) &&
            fwrite(&q, sizeof(chns_params), 1, fp) == 1;
  for (int k = 0; ok && k <= c->p.model; k++) ok = fwrite(f[k].data(), sizeof(double), f[k].size(), fp) == f[k].size();
  ok = (fclose(fp) == 0) && ok;
  return ok ? CHNS_OK : CHNS_ERR_IO;
}

int chns_load(chns_ctx* c, const char* path) {
  if (!c || !path) return CHNS_ERR_ARG;
  FILE* fp = fopen(path, "rb");
  if (!fp) return CHNS_ERR_IO;
  char magic[8];
  chns_params p;
  bool ok = fread(magic, 1, sizeof(magic), fp) == sizeof(magic) && memcmp(magic, kCkptMagic, sizeof(magic)) == 0 &&
            fread(&p, sizeof(p), 1, fp) == 1;
  if (!ok) {
    fclose(fp);
    return CHNS_ERR_IO;
  }
  const chns_params q = canonical(c->p), r = canonical(p);
  if (memcmp(&q, &r, sizeof(q)) != 0) {  // another configuration
    fclose(fp);
    return CHNS_ERR_ARG;
  }
  const size_t ncx = (size_t)c->n * c->nr;
  std::vector<double> f[3];
  for (int k = 0; ok && k <= c->p.model; k++) {
    f[k].resize(2 * ncx);
    ok = fread(f[k].data(), sizeof(double), f[k].size(), fp) == f[k].size();
  }
  fclose(fp);
  if (!ok) return CHNS_ERR_IO;
  return chns_set_state(c, f[0].data(), c->p.model >= 1 ? f[1].data() : nullptr,
                        c->p.model == 2 ? f[2].data() : nullptr, CHNS_HOST);
}

}  // extern "C"
