// `rang._core`: the gridder functions of the reference's PyO3 extension
// (core/py/src/lib.rs:1053-1446, registered at :2945-2950) with the same
// Python signatures, argument checks and status returns, bound to the C ABI
// of include/rang_wgridder.h. NumPy arrays are borrowed in place (C-contiguous
// only) and the GIL is released during each call. The `wgridder_plan_*`
// functions are this library's device-pointer extension.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <complex>
#include <string>
#include <vector>

#include "rang_weights.h"
#include "rang_wgridder.h"

namespace py = pybind11;

namespace {

// WgridderOptions from its 18 fields in declaration order (lib.rs:1053-1078).
WgridderOptions options(const std::vector<double>& o) {
  if (o.size() != 18) throw py::value_error("18 gridder options required");
  WgridderOptions w;
  w.nx = (size_t)o[0];
  w.ny = (size_t)o[1];
  w.pixsize_x = o[2];
  w.pixsize_y = o[3];
  w.epsilon = o[4];
  w.center_x = o[5];
  w.center_y = o[6];
  w.sigma_min = o[7];
  w.sigma_max = o[8];
  w.do_wgridding = (int32_t)o[9];
  w.divide_by_n = (int32_t)o[10];
  w.flip_u = (int32_t)o[11];
  w.flip_v = (int32_t)o[12];
  w.flip_w = (int32_t)o[13];
  w.allow_nshift = (int32_t)o[14];
  w.kernel_index = (int64_t)o[15];
  w.nu = (size_t)o[16];
  w.nv = (size_t)o[17];
  return w;
}

bool is_c(const py::array& a) { return (a.flags() & py::array::c_style) != 0; }

template <class T>
bool of_type(const py::array& a) {
  return py::dtype::of<T>().is(a.dtype()) || a.dtype().equal(py::dtype::of<T>());
}

// A read-only array of element type T, C-contiguous (lib.rs:114-139).
template <class T>
const T* ro(const py::object& o, const char* name, size_t* len) {
  py::array a = py::reinterpret_borrow<py::array>(o);
  if (!of_type<T>(a)) throw py::type_error(std::string(name) + " has the wrong dtype");
  if (!is_c(a)) throw py::value_error(std::string(name) + " must be C-contiguous");
  *len = (size_t)a.size();
  return static_cast<const T*>(a.data());
}

template <class T>
T* rw(const py::object& o, const char* name, size_t* len) {
  py::array a = py::reinterpret_borrow<py::array>(o);
  if (!of_type<T>(a)) throw py::type_error(std::string(name) + " has the wrong dtype");
  if (!is_c(a)) throw py::value_error(std::string(name) + " must be C-contiguous");
  if (!a.writeable()) throw py::value_error(std::string(name) + " must be writeable");
  *len = (size_t)a.size();
  return static_cast<T*>(a.mutable_data());
}

bool is_array(const py::object& o) { return !o.is_none() && py::isinstance<py::array>(o); }

// VisArg::extract (lib.rs:1090-1104).
const void* vis_arg(const py::object& o, int* kind, size_t* len) {
  *len = 0;
  if (o.is_none()) {
    *kind = WGRIDDER_VIS_UNIT;
    return nullptr;
  }
  if (!is_array(o)) throw py::value_error("vis must be complex64 or complex128");
  py::array a = py::reinterpret_borrow<py::array>(o);
  if (of_type<std::complex<float>>(a)) {
    *kind = WGRIDDER_VIS_C64;
    return ro<std::complex<float>>(o, "vis", len);
  }
  if (of_type<std::complex<double>>(a)) {
    *kind = WGRIDDER_VIS_C128;
    return ro<std::complex<double>>(o, "vis", len);
  }
  throw py::value_error("vis must be complex64 or complex128");
}

// WgtArg::extract (lib.rs:1129-1143).
const void* wgt_arg(const py::object& o, int* kind, size_t* len) {
  *len = 0;
  if (o.is_none()) {
    *kind = WGRIDDER_WGT_NONE;
    return nullptr;
  }
  if (!is_array(o)) throw py::value_error("weights must be float32 or float64");
  py::array a = py::reinterpret_borrow<py::array>(o);
  if (of_type<float>(a)) {
    *kind = WGRIDDER_WGT_F32;
    return ro<float>(o, "wgt", len);
  }
  if (of_type<double>(a)) {
    *kind = WGRIDDER_WGT_F64;
    return ro<double>(o, "wgt", len);
  }
  throw py::value_error("weights must be float32 or float64");
}

using V2d = int32_t (*)(const WgridderOptions*, size_t, size_t, const double*, const double*, const void*, int32_t,
                        const void*, const void*, int32_t, const uint8_t*, void*, void*, double*);

// wgridder_v2d (lib.rs:1193-1251).
template <class T>
int32_t v2d(const std::vector<double>& opts, const py::object& uvw, const py::object& freq, const py::object& vis,
            const py::object& wgt, const py::object& wgt2, const py::object& mask, const py::object& dirty,
            const py::object& psf, const py::object& info, V2d run) {
  WgridderOptions o = options(opts);
  size_t nuvw, nfreq, nvis = 0, nwgt = 0, nwgt2 = 0, nmask = 0, ndirty = 0, npsf = 0, ninfo;
  const double* puvw = ro<double>(uvw, "uvw", &nuvw);
  const double* pfreq = ro<double>(freq, "freq", &nfreq);
  size_t nrow = nuvw / 3, nchan = nfreq, n = nrow * nchan, npix = o.nx * o.ny;
  int vkind, wkind;
  const void* pvis = vis_arg(vis, &vkind, &nvis);
  const void* pwgt = wgt_arg(wgt, &wkind, &nwgt);
  const void* pwgt2 = nullptr;
  if (!wgt2.is_none()) {
    if (wkind != WGRIDDER_WGT_F32) throw py::value_error("two weights must both be float32");
    pwgt2 = ro<float>(wgt2, "wgt2", &nwgt2);
    wkind = WGRIDDER_WGT_F32_PRODUCT;
  }
  const uint8_t* pmask = mask.is_none() ? nullptr : ro<uint8_t>(mask, "mask", &nmask);
  T* pdirty = dirty.is_none() ? nullptr : rw<T>(dirty, "dirty", &ndirty);
  T* ppsf = psf.is_none() ? nullptr : rw<T>(psf, "psf", &npsf);
  double* pinfo = rw<double>(info, "info", &ninfo);
  bool ok = nuvw == nrow * 3 && (vis.is_none() || nvis == n) && (wgt.is_none() || nwgt == n) &&
            (wgt2.is_none() || nwgt2 == n) && (mask.is_none() || nmask == n) &&
            (dirty.is_none() || ndirty == npix) && (psf.is_none() || npsf == npix) && ninfo == 14;
  if (!ok) throw py::value_error("gridder array sizes disagree");
  py::gil_scoped_release release;
  return run(&o, nrow, nchan, puvw, pfreq, pvis, vkind, pwgt, pwgt2, wkind, pmask, pdirty, ppsf, pinfo);
}

using D2v = int32_t (*)(const WgridderOptions*, size_t, size_t, const double*, const double*, const void*,
                        const void*, int32_t, const uint8_t*, void*, double*);

// wgridder_d2v (lib.rs:1327-1367); `vis` is the real view (2 n values).
template <class T>
int32_t d2v(const std::vector<double>& opts, const py::object& uvw, const py::object& freq, const py::object& dirty,
            const py::object& wgt, const py::object& mask, const py::object& vis, const py::object& info, D2v run) {
  WgridderOptions o = options(opts);
  size_t nuvw, nfreq, ndirty, nwgt = 0, nmask = 0, nvis, ninfo;
  const double* puvw = ro<double>(uvw, "uvw", &nuvw);
  const double* pfreq = ro<double>(freq, "freq", &nfreq);
  size_t nrow = nuvw / 3, nchan = nfreq, n = nrow * nchan;
  const T* pdirty = ro<T>(dirty, "dirty", &ndirty);
  int wkind;
  const void* pwgt = wgt_arg(wgt, &wkind, &nwgt);
  const uint8_t* pmask = mask.is_none() ? nullptr : ro<uint8_t>(mask, "mask", &nmask);
  T* pvis = rw<T>(vis, "vis", &nvis);
  double* pinfo = rw<double>(info, "info", &ninfo);
  bool ok = nuvw == nrow * 3 && ndirty == o.nx * o.ny && nvis == 2 * n && (wgt.is_none() || nwgt == n) &&
            (mask.is_none() || nmask == n) && ninfo == 14;
  if (!ok) throw py::value_error("gridder array sizes disagree");
  py::gil_scoped_release release;
  return run(&o, nrow, nchan, puvw, pfreq, pdirty, pwgt, wkind, pmask, pvis, pinfo);
}

int32_t v2d_f64(const WgridderOptions* o, size_t r, size_t c, const double* u, const double* f, const void* v, int32_t vk,
                const void* w, const void* w2, int32_t wk, const uint8_t* m, void* d, void* p, double* i) {
  return rang_core_wgridder_vis2dirty_ex2_f64(o, r, c, u, f, v, vk, w, w2, wk, m, (double*)d, (double*)p, i);
}
int32_t v2d_f32(const WgridderOptions* o, size_t r, size_t c, const double* u, const double* f, const void* v, int32_t vk,
                const void* w, const void* w2, int32_t wk, const uint8_t* m, void* d, void* p, double* i) {
  return rang_core_wgridder_vis2dirty_ex2_f32(o, r, c, u, f, v, vk, w, w2, wk, m, (float*)d, (float*)p, i);
}
int32_t d2v_f64(const WgridderOptions* o, size_t r, size_t c, const double* u, const double* f, const void* d,
                const void* w, int32_t wk, const uint8_t* m, void* v, double* i) {
  return rang_core_wgridder_dirty2vis_ex_f64(o, r, c, u, f, (const double*)d, w, wk, m, (double*)v, i);
}
int32_t d2v_f32(const WgridderOptions* o, size_t r, size_t c, const double* u, const double* f, const void* d,
                const void* w, int32_t wk, const uint8_t* m, void* v, double* i) {
  return rang_core_wgridder_dirty2vis_ex_f32(o, r, c, u, f, (const float*)d, w, wk, m, (float*)v, i);
}

std::string last_error() {
  size_t n = rang_core_wgridder_last_error(nullptr, 0);
  std::string s(n, '\0');
  rang_core_wgridder_last_error(reinterpret_cast<uint8_t*>(s.data()), n);
  return s;
}

const void* ptr(uintptr_t p) { return reinterpret_cast<const void*>(p); }

}  // namespace

PYBIND11_MODULE(_core, m) {
  m.doc() = "rang._core: the B200 w-gridder behind the reference's Python-level gridder functions";
  m.def(
      "wgridder_vis2dirty_f64",
      [](std::vector<double> opts, py::object uvw, py::object freq, py::object vis, py::object wgt, py::object wgt2,
         py::object mask, py::object dirty, py::object psf, py::object info) {
        return v2d<double>(opts, uvw, freq, vis, wgt, wgt2, mask, dirty, psf, info, v2d_f64);
      },
      py::arg("opts"), py::arg("uvw"), py::arg("freq"), py::arg("vis"), py::arg("wgt"), py::arg("wgt2"),
      py::arg("mask"), py::arg("dirty"), py::arg("psf"), py::arg("info"));
  m.def(
      "wgridder_vis2dirty_f32",
      [](std::vector<double> opts, py::object uvw, py::object freq, py::object vis, py::object wgt, py::object wgt2,
         py::object mask, py::object dirty, py::object psf, py::object info) {
        return v2d<float>(opts, uvw, freq, vis, wgt, wgt2, mask, dirty, psf, info, v2d_f32);
      },
      py::arg("opts"), py::arg("uvw"), py::arg("freq"), py::arg("vis"), py::arg("wgt"), py::arg("wgt2"),
      py::arg("mask"), py::arg("dirty"), py::arg("psf"), py::arg("info"));
  m.def(
      "wgridder_dirty2vis_f64",
      [](std::vector<double> opts, py::object uvw, py::object freq, py::object dirty, py::object wgt, py::object mask,
         py::object vis, py::object info) { return d2v<double>(opts, uvw, freq, dirty, wgt, mask, vis, info, d2v_f64); },
      py::arg("opts"), py::arg("uvw"), py::arg("freq"), py::arg("dirty"), py::arg("wgt"), py::arg("mask"),
      py::arg("vis"), py::arg("info"));
  m.def(
      "wgridder_dirty2vis_f32",
      [](std::vector<double> opts, py::object uvw, py::object freq, py::object dirty, py::object wgt, py::object mask,
         py::object vis, py::object info) { return d2v<float>(opts, uvw, freq, dirty, wgt, mask, vis, info, d2v_f32); },
      py::arg("opts"), py::arg("uvw"), py::arg("freq"), py::arg("dirty"), py::arg("wgt"), py::arg("mask"),
      py::arg("vis"), py::arg("info"));
  m.def("wgridder_kernel_row", [](size_t index, py::object out) {
    size_t n;
    double* p = rw<double>(out, "out", &n);
    if (n != 7) return 1;
    return (int)rang_core_wgridder_kernel_row(index, p);
  });
  m.def("wgridder_last_error", &last_error);

  // Imaging weights and Stokes I (lib.rs:792-904): the reference's bindings of ffi_weights.rs.
  m.def("weight_grid_shape", [](size_t width, size_t height, double super_weight) {
    size_t shape[2] = {0, 0};
    int st = (int)rang_core_weight_grid_shape(width, height, super_weight, shape);
    return py::make_tuple(st, shape[0], shape[1]);
  });
  m.def("padded_size", [](size_t trimmed, double padding) { return rang_core_padded_size(trimmed, padding); });
  m.def("stokes_i", [](size_t ncell, py::object data, py::object weights, py::object flags, py::object vis,
                       py::object weight) {
    size_t nd, nw, nf, nv, no;
    StokesIInputs in{ncell, ro<float>(data, "data", &nd), ro<float>(weights, "weights", &nw),
                     ro<uint8_t>(flags, "flags", &nf)};
    StokesIOutputs out{rw<float>(vis, "vis", &nv), rw<float>(weight, "weight", &no)};
    if (nd != 8 * ncell) throw py::value_error("data must hold 8 * ncell floats");
    if (nw != 4 * ncell || nf != 4 * ncell) throw py::value_error("weights and flags must hold 4 * ncell values");
    if (nv != 2 * ncell || no != ncell) throw py::value_error("vis must hold 2 * ncell and weight ncell values");
    py::gil_scoped_release release;
    return (int)rang_core_stokes_i(&in, &out);
  });
  m.def("imaging_weights",
        [](size_t nrow, size_t nchan, py::object uvw, py::object wavelength, py::object weights,
           py::object row_selected, uint32_t cls, double robust, size_t width, size_t height, double psx, double psy,
           double super_weight, double level, size_t rank_size, py::object out_weights, py::object grid,
           py::object sums) {
          size_t nu, nl, nw, ns, no, ng = 0, nsum = 0;
          ImagingWeightInputs in{};
          in.nrow = nrow;
          in.nchan = nchan;
          in.uvw = ro<double>(uvw, "uvw", &nu);
          in.wavelength = ro<double>(wavelength, "wavelength", &nl);
          in.weights = ro<float>(weights, "weights", &nw);
          in.row_selected = ro<uint8_t>(row_selected, "row_selected", &ns);
          in.class_ = cls;
          in.robust = robust;
          in.width = width;
          in.height = height;
          in.pixel_scale_x = psx;
          in.pixel_scale_y = psy;
          in.super_weight = super_weight;
          in.rank_filter_level = level;
          in.rank_filter_size = rank_size;
          if (nu != 3 * nrow) throw py::value_error("uvw must hold 3 * nrow values");
          if (nl != nchan) throw py::value_error("wavelength must hold nchan values");
          if (nw != nrow * nchan) throw py::value_error("weights must hold nrow * nchan values");
          if (ns != nrow) throw py::value_error("row_selected must hold nrow values");
          ImagingWeightOutputs out{};
          out.weights = rw<float>(out_weights, "out_weights", &no);
          if (no != nrow * nchan) throw py::value_error("out_weights must hold nrow * nchan values");
          if (!grid.is_none()) {
            out.grid = rw<double>(grid, "grid", &ng);
            if (super_weight > 0.0) {
              size_t shape[2];
              rang_core_weight_grid_shape(width, height, super_weight, shape);
              if (ng != shape[0] * shape[1] / 2) throw py::value_error("grid must hold width * height / 2 values");
            }
          }
          if (!sums.is_none()) {
            out.sums = rw<double>(sums, "sums", &nsum);
            if (nsum != 4) throw py::value_error("sums must hold 4 values");
          }
          py::gil_scoped_release release;
          return (int)rang_core_imaging_weights(&in, &out);
        },
        py::arg("nrow"), py::arg("nchan"), py::arg("uvw"), py::arg("wavelength"), py::arg("weights"),
        py::arg("row_selected"), py::arg("class_"), py::arg("robust"), py::arg("width"), py::arg("height"),
        py::arg("pixel_scale_x"), py::arg("pixel_scale_y"), py::arg("super_weight"), py::arg("rank_filter_level"),
        py::arg("rank_filter_size"), py::arg("out_weights"), py::arg("grid"), py::arg("sums"));

  // Device-pointer plans (pointers as integers, e.g. torch.Tensor.data_ptr()).
  m.def(
      "wgridder_plan_create",
      [](std::vector<double> opts, size_t nrow, size_t nchan, uintptr_t uvw, py::array_t<double> freq, uintptr_t vis,
         int vis_kind, uintptr_t wgt, uintptr_t wgt2, int wgt_kind, uintptr_t mask, int with_vis, int single,
         uintptr_t stream) {
        WgridderOptions o = options(opts);
        if ((size_t)freq.size() != nchan) throw py::value_error("freq must have nchan values");
        py::array_t<double> info(14);
        RangWgridPlan* plan = nullptr;
        int32_t st;
        {
          py::gil_scoped_release release;
          st = rang_b200_wgridder_plan_create(&o, nrow, nchan, (const double*)ptr(uvw), freq.data(), ptr(vis),
                                              vis_kind, ptr(wgt), ptr(wgt2), wgt_kind, (const uint8_t*)ptr(mask),
                                              with_vis, single, (void*)stream, &plan, info.mutable_data());
        }
        return py::make_tuple(st, reinterpret_cast<uintptr_t>(plan), info);
      });
  m.def("wgridder_plan_grid", [](uintptr_t plan, uintptr_t vis, int vis_kind, uintptr_t wgt, uintptr_t wgt2,
                                 int wgt_kind, int flags, uintptr_t image, uintptr_t stream) {
    py::gil_scoped_release release;
    return rang_b200_wgridder_plan_grid(reinterpret_cast<RangWgridPlan*>(plan), ptr(vis), vis_kind, ptr(wgt),
                                        ptr(wgt2), wgt_kind, flags, (void*)image, (void*)stream);
  });
  m.def("wgridder_plan_degrid",
        [](uintptr_t plan, uintptr_t image, uintptr_t wgt, int wgt_kind, uintptr_t vis, uintptr_t stream) {
          py::gil_scoped_release release;
          return rang_b200_wgridder_plan_degrid(reinterpret_cast<RangWgridPlan*>(plan), ptr(image), ptr(wgt),
                                                wgt_kind, (void*)vis, (void*)stream);
        });
  m.def("wgridder_plan_status", [](uintptr_t plan, uintptr_t stream) {
    py::gil_scoped_release release;
    return rang_b200_wgridder_plan_status(reinterpret_cast<RangWgridPlan*>(plan), (void*)stream);
  });
  m.def("wgridder_plan_destroy", [](uintptr_t plan) {
    py::gil_scoped_release release;
    rang_b200_wgridder_plan_destroy(reinterpret_cast<RangWgridPlan*>(plan));
  });
  m.def("wgridder_plan_residual",
        [](uintptr_t plan, uintptr_t data, int vis_kind, uintptr_t wgt, uintptr_t wgt2, int wgt_kind, uintptr_t model,
           int sorted, uintptr_t image, uintptr_t misfit, uintptr_t stream) {
          py::gil_scoped_release release;
          return rang_b200_wgridder_plan_residual(reinterpret_cast<RangWgridPlan*>(plan), ptr(data), vis_kind,
                                                  ptr(wgt), ptr(wgt2), wgt_kind, ptr(model), sorted, (void*)image,
                                                  (double*)misfit, (void*)stream);
        });
  m.def("wgridder_plan_gram", [](uintptr_t plan, uintptr_t x, uintptr_t wgt, uintptr_t wgt2, int wgt_kind, int sorted,
                                 uintptr_t image, uintptr_t xgx, uintptr_t stream) {
    py::gil_scoped_release release;
    return rang_b200_wgridder_plan_gram(reinterpret_cast<RangWgridPlan*>(plan), ptr(x), ptr(wgt), ptr(wgt2), wgt_kind,
                                        sorted, (void*)image, (double*)xgx, (void*)stream);
  });
  m.def("wgridder_plan_sorted", [](uintptr_t plan, uintptr_t dense, int elem_bytes, uintptr_t out, uintptr_t stream) {
    py::gil_scoped_release release;
    return rang_b200_wgridder_plan_sorted(reinterpret_cast<RangWgridPlan*>(plan), ptr(dense), elem_bytes,
                                          (void*)out, (void*)stream);
  });
  m.def("wgridder_plan_active", [](uintptr_t plan) {
    size_t n = 0;
    int st = rang_b200_wgridder_plan_active(reinterpret_cast<RangWgridPlan*>(plan), &n);
    return py::make_tuple(st, n);
  });
  m.def("wgridder_plan_memory", [](uintptr_t plan) {
    size_t b[32];
    int n = rang_b200_wgridder_plan_memory(reinterpret_cast<RangWgridPlan*>(plan), b, 32);
    py::list out;
    for (int i = 0; i < n && i < 32; i++)
      out.append(py::make_tuple(std::string(rang_b200_wgridder_plan_memory_name(i)), b[i]));
    return out;
  });
  m.def("wgridder_cached_bytes", []() { return rang_b200_wgridder_cached_bytes(); });
  m.def("wgridder_release_cached", []() { return rang_b200_wgridder_release_cached(); });
  m.def("wgridder_plan_release_work",
        [](uintptr_t plan) { rang_b200_wgridder_plan_release_work(reinterpret_cast<RangWgridPlan*>(plan)); });
  m.def("wgridder_plan_only", [](std::vector<double> opts, py::object uvw, py::object freq, py::object vis,
                                 py::object wgt, py::object wgt2, py::object mask, int single, int nout) {
    WgridderOptions o = options(opts);
    size_t nuvw, nfreq, nvis = 0, nwgt = 0, nwgt2 = 0, nmask = 0;
    const double* puvw = ro<double>(uvw, "uvw", &nuvw);
    const double* pfreq = ro<double>(freq, "freq", &nfreq);
    int vkind, wkind;
    const void* pvis = vis_arg(vis, &vkind, &nvis);
    const void* pwgt = wgt_arg(wgt, &wkind, &nwgt);
    const void* pwgt2 = nullptr;
    if (!wgt2.is_none()) {
      pwgt2 = ro<float>(wgt2, "wgt2", &nwgt2);
      wkind = WGRIDDER_WGT_F32_PRODUCT;
    }
    const uint8_t* pmask = mask.is_none() ? nullptr : ro<uint8_t>(mask, "mask", &nmask);
    py::array_t<double> info(14);
    size_t fp = 0;
    int32_t st;
    {
      py::gil_scoped_release release;
      st = rang_b200_wgridder_plan_only(&o, nuvw / 3, nfreq, puvw, pfreq, pvis, vkind, pwgt, pwgt2, wkind, pmask,
                                        single, nout, info.mutable_data(), &fp);
    }
    return py::make_tuple(st, info, fp);
  });
  m.def("wgridder_set_method", [](int m) { return (int)rang_b200_wgridder_set_method(m); });
  m.def("wgridder_launch_count", []() { return (long long)rang_b200_wgridder_launch_count(); });
  m.def("wgridder_profile", [](int on) { rang_b200_wgridder_profile(on); });
  m.def("wgridder_profile_read", []() {
    int64_t l[64];
    double t[64];
    int n;
    {
      py::gil_scoped_release release;
      n = rang_b200_wgridder_profile_read(l, t, 64);
    }
    py::dict out;
    for (int i = 0; i < n; i++) out[py::str(rang_b200_wgridder_stage_name(i))] = py::make_tuple(l[i], t[i]);
    return out;
  });
  m.def(
      "wgridder_binning",
      [](std::vector<double> opts, py::object uvw, py::object freq, py::object vis, py::object wgt, py::object wgt2,
         py::object mask, int with_vis, int single) {
        WgridderOptions o = options(opts);
        size_t nuvw, nfreq, nvis = 0, nwgt = 0, nwgt2 = 0, nmask = 0;
        const double* puvw = ro<double>(uvw, "uvw", &nuvw);
        const double* pfreq = ro<double>(freq, "freq", &nfreq);
        size_t nrow = nuvw / 3, nchan = nfreq, n = nrow * nchan;
        int vkind, wkind;
        const void* pvis = vis_arg(vis, &vkind, &nvis);
        const void* pwgt = wgt_arg(wgt, &wkind, &nwgt);
        const void* pwgt2 = nullptr;
        if (!wgt2.is_none()) {
          pwgt2 = ro<float>(wgt2, "wgt2", &nwgt2);
          wkind = WGRIDDER_WGT_F32_PRODUCT;
        }
        const uint8_t* pmask = mask.is_none() ? nullptr : ro<uint8_t>(mask, "mask", &nmask);
        py::array_t<int64_t> iu0(n), iv0(n);
        py::array_t<uint32_t> key(n), sorted(n);
        py::array_t<double> info(14);
        size_t ns = 0;
        int32_t st;
        {
          py::gil_scoped_release release;
          st = rang_b200_wgridder_binning(&o, nrow, nchan, puvw, pfreq, pvis, vkind, pwgt, pwgt2, wkind, pmask,
                                          with_vis, single, iu0.mutable_data(), iv0.mutable_data(),
                                          key.mutable_data(), sorted.mutable_data(), &ns, info.mutable_data());
        }
        return py::make_tuple(st, iu0, iv0, key, sorted, ns, info);
      });
}
