// chns_io.cu -- field files in the reference's format (write_array.c, read_array.c).
//
// Raw FP64 nx x ny arrays, row-major with x the slow index and no header: the
// layout write_array_real produces after gathering the slabs (write_array.c:18-46)
// and read_array_real consumes (read_array.c:12-40).  The real-space fields are
// computed on the device (ifft, optionally after truncation) and written by the host.
#include <cuda_runtime.h>
#include <errno.h>
#include <stdio.h>
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

}  // extern "C"
