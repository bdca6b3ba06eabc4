// Test infrastructure (never linked into the product): a C-ABI shim around the
// reference's own histogram I/O (cpp/histogramIO.h, which reads and writes PNM
// through the vendored CImg without ImageMagick), so that the golden fixtures
// for histio.py come from the reference's code.  Built by oracle/Makefile into
// oracle/_ref/libhistioref.so from the unmodified reference sources.
#include <cstring>
#include <string>
#include <vector>

#include "histogramIO.h"

extern "C" {

// load_img_to_pdf (cpp/histogramIO.h:243-259); returns the sum, W and H.
double href_load_img_to_pdf(const char* fn, double* out, int cap, int* W, int* H) {
  std::vector<double> r;
  const double s = load_img_to_pdf(fn, r, *W, *H);
  std::memcpy(out, r.data(), sizeof(double) * (r.size() < (size_t)cap ? r.size() : (size_t)cap));
  return s;
}

// load_rgb_img_to_pdf_grayscale_luma (:269-285)
double href_load_rgb_luma(const char* fn, double* out, int cap, int* W, int* H) {
  std::vector<double> r;
  const double s = load_rgb_img_to_pdf_grayscale_luma(fn, r, *W, *H);
  std::memcpy(out, r.data(), sizeof(double) * (r.size() < (size_t)cap ? r.size() : (size_t)cap));
  return s;
}

// load_img_to_pdf_gamma_correction (:287-312)
double href_load_gamma(const char* fn, double* out, int cap, int* W, int* H, double alpha, int complement) {
  std::vector<double> r;
  const double s = load_img_to_pdf_gamma_correction(fn, r, *W, *H, alpha, complement != 0);
  std::memcpy(out, r.data(), sizeof(double) * (r.size() < (size_t)cap ? r.size() : (size_t)cap));
  return s;
}

// load_csv_to_pdf (:314-337); returns the number of values.
int href_load_csv(const char* fn, double* out, int cap, double* sum) {
  std::vector<double> r;
  *sum = load_csv_to_pdf(fn, r);
  std::memcpy(out, r.data(), sizeof(double) * (r.size() < (size_t)cap ? r.size() : (size_t)cap));
  return (int)r.size();
}

// save_pdf (:339-351) and save_pdf_gamma_correction (:353-371)
void href_save_pdf(const char* fn, int W, int H, const double* val, double scaling) {
  save_pdf(fn, W, H, std::vector<double>(val, val + (size_t)W * H), scaling);
}
void href_save_pdf_gamma(const char* fn, int W, int H, const double* val, double alpha, int complement,
                         double scaling) {
  save_pdf_gamma_correction(fn, W, H, std::vector<double>(val, val + (size_t)W * H), alpha, complement != 0,
                            scaling);
}

// quantile (:379-405)
void href_quantile(const double* data, int n, const double* probs, int np, double* out) {
  const std::vector<double> q = quantile(std::vector<double>(data, data + n), std::vector<double>(probs, probs + np));
  for (int i = 0; i < np; ++i) out[i] = q[i];
}

}  // extern "C"
