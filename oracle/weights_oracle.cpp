// CPU ORACLE — test infrastructure only, never shipped or called by the product.
//
// A sequential C++ restatement of the reference's imaging-weight path,
// `core/src/weights.rs` (rang-core's port of WSClean 3.6's
// `structures/imageweights.cpp`: half-plane weight grid, Briggs / uniform /
// natural finish, rank filter, nearest-cell lookup, Stokes I formation and
// the header sums). Every function names the reference lines it restates and
// keeps their floating-point order (float weights accumulated in doubles in
// row and channel order), so the results are the reference's bit for bit.
// Only the tests load it, through oracle.py.

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace {

// WeightGrid::shape (weights.rs:102-112).
void grid_shape(size_t width, size_t height, double super_weight, size_t* w, size_t* h) {
  size_t a = (size_t)std::llround((double)width / super_weight);
  size_t b = (size_t)std::llround((double)height / super_weight);
  // Rust's f64::round rounds half away from zero, as llround does.
  if (a % 2) a++;
  if (b % 2) b++;
  *w = a;
  *h = b;
}

struct Grid {
  size_t width = 0, height = 0;
  double scale_x = 0, scale_y = 0;
  std::vector<double> cells;
  double total = 0;

  // uv_to_xy (weights.rs:131-140).
  void uv_to_xy(double u, double v, int64_t* x, int64_t* y) const {
    if (v < 0.0) {
      u = -u;
      v = -v;
    }
    *x = (int64_t)std::floor(u * (double)width * scale_x + (double)(width / 2));
    *y = (int64_t)std::floor(v * (double)height * scale_y);
  }
  // within (weights.rs:142-144).
  bool within(int64_t x, int64_t y) const {
    return x >= 0 && x < (int64_t)width && y < (int64_t)(height / 2);
  }
  // grid_sample (weights.rs:147-153).
  void sample_add(double u, double v, float weight) {
    int64_t x, y;
    uv_to_xy(u, v, &x, &y);
    if (within(x, y)) {
      cells[(size_t)x + (size_t)y * width] += (double)weight;
      total += (double)weight;
    }
  }
  // sample (weights.rs:271-278).
  double sample(double u, double v) const {
    int64_t x, y;
    uv_to_xy(u, v, &x, &y);
    return within(x, y) ? cells[(size_t)x + (size_t)y * width] : 0.0;
  }
  // window_mean (weights.rs:229-250).
  double window_mean(size_t x, size_t y, size_t window) const {
    size_t d = window / 2, half = height / 2;
    size_t x1 = x >= d ? x - d : 0, y1 = y >= d ? y - d : 0;
    size_t x2 = x + d >= width ? width : x + d;
    size_t y2 = y + d >= half ? half : y + d;
    size_t count = 0;
    double sum = 0.0;
    for (size_t yi = y1; yi < y2; yi++)
      for (size_t xi = x1; xi < x2; xi++) {
        double w = cells[yi * width + xi];
        if (w != 0.0) {
          count++;
          sum += w;
        }
      }
    return sum / (double)count;
  }
};

}  // namespace

extern "C" {

// padded_size (weights.rs:38-42).
size_t oracle_padded_size(size_t trimmed, double padding) {
  size_t padded = (size_t)std::ceil((double)trimmed * padding);
  padded += (4 - (padded % 4)) % 4;
  return padded;
}

void oracle_weight_grid_shape(size_t width, size_t height, double super_weight, size_t* shape) {
  grid_shape(width, height, super_weight, &shape[0], &shape[1]);
}

// stokes_i_from_linear (weights.rs:522-562).
void oracle_stokes_i(size_t ncell, const float* data, const float* weights, const uint8_t* flags, float* vis,
                     float* out) {
  auto finite = [](float a, float b) { return std::isfinite(a) && std::isfinite(b); };
  for (size_t c = 0; c < ncell; c++) {
    const float* d = data + 8 * c;
    float xx_re = d[0], xx_im = d[1], yy_re = d[6], yy_im = d[7];
    float re = (yy_re + xx_re) * 0.5f, im = (yy_im + xx_im) * 0.5f;
    vis[2 * c] = 0.0f;
    vis[2 * c + 1] = 0.0f;
    if (finite(re, im)) {
      vis[2 * c] = re;
      vis[2 * c + 1] = im;
    }
    const float* w = weights + 4 * c;
    const uint8_t* f = flags + 4 * c;
    float weight = (f[0] == 0 && finite(xx_re, xx_im)) ? w[0] * 4.0f : 0.0f;
    if (f[3] == 0 && finite(yy_re, yy_im)) {
      float yy = w[3] * 4.0f;
      weight = yy < weight ? yy : weight;
    } else {
      weight = 0.0f;
    }
    out[c] = weight;
  }
}

// imaging_weights_tapered without tapers (weights.rs:465-520): grid_rows
// (:158-188), finish (:190-227), rank_filter (:254-269), lookup_rows
// (:283-315), and weight_sums (:564-582). Returns 0, or 1 for invalid
// arguments as WeightGrid::new (:72-100) and the FFI (ffi_weights.rs:166-233).
int oracle_imaging_weights(size_t nrow, size_t nchan, const double* uvw, const double* wavelength,
                           const float* weights, const uint8_t* selected, uint32_t cls, double robust, size_t width,
                           size_t height, double scale_x, double scale_y, double super_weight, double rank_level,
                           size_t rank_size, float* out, double* grid_out, double* sums) {
  if (cls > 2) return 1;
  if (width == 0 || height == 0 || !(super_weight > 0.0) || scale_x <= 0.0 || scale_y <= 0.0) return 1;
  Grid g;
  grid_shape(width, height, super_weight, &g.width, &g.height);
  g.scale_x = scale_x;
  g.scale_y = scale_y;
  g.cells.assign(g.width * g.height / 2, 0.0);
  for (size_t row = 0; row < nrow; row++) {
    if (!selected[row]) continue;
    double um = uvw[3 * row], vm = uvw[3 * row + 1];
    if (vm < 0.0) {
      um = -um;
      vm = -vm;
    }
    for (size_t ch = 0; ch < nchan; ch++) g.sample_add(um / wavelength[ch], vm / wavelength[ch], weights[row * nchan + ch]);
  }
  if (cls == 2) {
    double avg_w = 0.0;
    for (double v : g.cells) avg_w += v * v;
    avg_w /= g.total;
    double numerator_sqrt = 5.0 * std::exp(-2.302585092994046 * robust);  // -LN_10 * robust
    double s_sq = numerator_sqrt * numerator_sqrt / avg_w;
    for (double& v : g.cells)
      if (v != 0.0) v = 1.0 / (1.0 + v * s_sq);
  } else if (cls == 1) {
    for (double& v : g.cells)
      if (v != 0.0) v = 1.0 / v;
  } else {
    for (double& v : g.cells)
      if (v != 0.0) v = 1.0;
  }
  if (rank_level >= 1.0) {
    std::vector<double> next = g.cells;
    for (size_t y = 0; y < g.height / 2; y++)
      for (size_t x = 0; x < g.width; x++) {
        double w = g.cells[y * g.width + x];
        if (w != 0.0) {
          double mean = g.window_mean(x, y, rank_size);
          if (w > mean * rank_level) next[y * g.width + x] = mean * rank_level;
        }
      }
    g.cells.swap(next);
  }
  for (size_t row = 0; row < nrow; row++)
    for (size_t ch = 0; ch < nchan; ch++) {
      float v = 0.0f;
      if (selected[row]) v = (float)g.sample(uvw[3 * row] / wavelength[ch], uvw[3 * row + 1] / wavelength[ch]);
      out[row * nchan + ch] = v;
    }
  if (grid_out)
    for (size_t i = 0; i < g.cells.size(); i++) grid_out[i] = g.cells[i];
  if (sums) {
    double vsum = 0.0, total = 0.0, largest = 0.0;
    uint64_t count = 0;
    for (size_t i = 0; i < nrow * nchan; i++) {
      float cum = weights[i] * out[i];
      if (cum != 0.0f) {
        vsum += (double)weights[i];
        count++;
      }
      largest = std::fmax(largest, (double)cum);
      total += (double)cum;
    }
    sums[0] = vsum;
    sums[1] = total;
    sums[2] = largest;
    sums[3] = (double)count;
  }
  return 0;
}

}  // extern "C"
