// _wolfgang_core: Python bindings of the drop-in classes (pybind11).
//
// Mirrors the names, keyword arguments, return shapes and exception types of
// the reference's nanobind module (bindings/python/pauli_sum_py.cpp:1036-1632,
// python/wolfgang_quantum/_wolfgang_core.pyi): std::invalid_argument ->
// ValueError, std::runtime_error -> RuntimeError, dtype/layout problems ->
// TypeError.  nanobind is not available in this toolchain; pybind11 provides the
// same Python-visible surface.

#include <pybind11/complex.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <bit>
#include <complex>
#include <cstring>
#include <limits>
#include <memory>
#include <span>
#include <string>
#include <vector>

#include "ATen/dlpack.h"  // the DLPack C ABI (a plain C header shipped with torch; no torch code)
#include "wg_pauli.h"
#include "wolfgang/device_pauli_sum.hpp"
#include "wolfgang/pauli_sum.hpp"

namespace py = pybind11;
using namespace wolfgang;

namespace {

[[noreturn]] void value_error(const std::string& m) { throw py::value_error(m); }
[[noreturn]] void type_error(const std::string& m) { throw py::type_error(m); }

std::size_t size_arg(const py::handle& v, const char* name) {
  if (!PyLong_Check(v.ptr())) value_error(std::string(name) + " must be a non-negative integer");
  const unsigned long long raw = PyLong_AsUnsignedLongLong(v.ptr());
  if (PyErr_Occurred()) {
    PyErr_Clear();
    value_error(std::string(name) + " must be a non-negative integer that fits size_t");
  }
  return static_cast<std::size_t>(raw);
}

std::size_t nonneg(long long v, const char* name) {
  if (v < 0) value_error(std::string(name) + " must be non-negative");
  return static_cast<std::size_t>(v);
}

template <typename F>
auto translate(F&& f) -> decltype(f()) {
  try {
    return f();
  } catch (const std::invalid_argument& e) {
    throw py::value_error(e.what());
  }
}

std::complex<double> complex_arg(const py::handle& v, const char* name) {
  if (PyComplex_Check(v.ptr())) return {PyComplex_RealAsDouble(v.ptr()), PyComplex_ImagAsDouble(v.ptr())};
  if (PyFloat_Check(v.ptr()) || PyLong_Check(v.ptr()) || PyIndex_Check(v.ptr()) ||
      py::hasattr(v, "__complex__") || py::hasattr(v, "__float__")) {
    const Py_complex c = PyComplex_AsCComplex(v.ptr());
    if (!PyErr_Occurred()) return {c.real, c.imag};
    PyErr_Clear();
  }
  value_error(std::string(name) + " must be numeric");
}

bool is_numeric_scalar(const py::handle& v) {
  if (PyUnicode_Check(v.ptr()) || PyBytes_Check(v.ptr())) return false;
  if (PyComplex_Check(v.ptr()) || PyFloat_Check(v.ptr()) || PyLong_Check(v.ptr())) return true;
  if (py::isinstance<py::array>(v)) return py::reinterpret_borrow<py::array>(v).ndim() == 0;
  return py::hasattr(v, "__complex__") || py::hasattr(v, "__float__");
}

std::vector<std::string> parse_labels(const py::handle& labels) {
  if (PyUnicode_Check(labels.ptr()))
    value_error("labels must be an iterable of dense label strings, not a single string");
  std::vector<std::string> out;
  try {
    for (py::handle item : py::iter(labels)) {
      if (!PyUnicode_Check(item.ptr())) value_error("labels must be an iterable of strings");
      out.push_back(item.cast<std::string>());
    }
  } catch (const py::error_already_set&) {
    value_error("labels must be an iterable of strings");
  }
  return out;
}

std::vector<std::complex<double>> parse_coeffs(const py::object& coeffs, std::size_t n) {
  if (coeffs.is_none()) return std::vector<std::complex<double>>(n, {1.0, 0.0});
  if (is_numeric_scalar(coeffs)) {
    if (n != 1) value_error("scalar coeffs are valid only for a single label");
    return {complex_arg(coeffs, "coefficients")};
  }
  std::vector<std::complex<double>> out;
  try {
    for (py::handle item : py::iter(coeffs)) out.push_back(complex_arg(item, "coefficients"));
  } catch (const py::error_already_set&) {
    value_error("coeffs must be None, a numeric scalar for one label, or an iterable of numeric values");
  }
  if (out.size() != n) value_error("coefficient count must match label count");
  return out;
}

std::vector<PauliSum::SparseTerm> parse_sparse(const py::handle& triples) {
  std::vector<PauliSum::SparseTerm> out;
  for (py::handle item : py::iter(triples)) {
    if (!PySequence_Check(item.ptr()) || PyUnicode_Check(item.ptr()) || PySequence_Size(item.ptr()) != 3)
      value_error("each sparse term must be a 3-item sequence");
    py::sequence seq = py::reinterpret_borrow<py::sequence>(item);
    PauliSum::SparseTerm t;
    if (!PyUnicode_Check(seq[0].ptr())) value_error("sparse local_pauli_string must be a string");
    t.local_pauli_string = seq[0].cast<std::string>();
    py::object idx = seq[1];
    if (!PySequence_Check(idx.ptr()) || PyUnicode_Check(idx.ptr()))
      value_error("qubit_indices must be a sequence of non-negative integers");
    for (py::handle q : py::reinterpret_borrow<py::sequence>(idx)) {
      if (!PyLong_Check(q.ptr()) && !PyIndex_Check(q.ptr())) value_error("qubit_indices must contain integers");
      const long long v = PyLong_AsLongLong(q.ptr());
      if (PyErr_Occurred()) {
        PyErr_Clear();
        value_error("qubit_indices must contain integers");
      }
      if (v < 0) value_error("qubit_indices must be a sequence of non-negative integers");
      t.qubit_indices.push_back(static_cast<std::size_t>(v));
    }
    t.coefficient = complex_arg(seq[2], "coefficient");
    out.push_back(std::move(t));
  }
  return out;
}

py::array_t<std::complex<double>> coeff_array(const std::vector<std::complex<double>>& c) {
  py::array_t<std::complex<double>> a(static_cast<py::ssize_t>(c.size()));
  if (!c.empty()) std::memcpy(a.mutable_data(), c.data(), c.size() * sizeof(std::complex<double>));
  return a;
}

py::array bool_array(const std::vector<std::uint8_t>& flags) {
  py::array_t<bool> a(static_cast<py::ssize_t>(flags.size()));
  if (!flags.empty()) std::memcpy(a.mutable_data(), flags.data(), flags.size());
  return a;
}

py::array u64_array(const std::vector<std::uint64_t>& v) {
  py::array_t<std::uint64_t> a(static_cast<py::ssize_t>(v.size()));
  if (!v.empty()) std::memcpy(a.mutable_data(), v.data(), v.size() * 8);
  return a;
}

// bool scalar / 1-D / 2-D shaping of the reference (pauli_sum_py.cpp:1194-1222).
py::object shape_flags(const std::vector<std::uint8_t>& flags, std::size_t l, std::size_t r) {
  if (l == 1 && r == 1) return py::bool_(!flags.empty() && flags.front() != 0);
  py::array a = bool_array(flags);
  if (l == 1 || r == 1) return a;
  return a.reshape({static_cast<py::ssize_t>(l), static_cast<py::ssize_t>(r)});
}

// Host statevector through the buffer protocol (pauli_sum_py.cpp:334-371).
template <typename Op>
py::object host_expectation(const Op& op, const py::handle& psi_obj) {
  py::buffer_info info;
  try {
    info = py::reinterpret_borrow<py::buffer>(psi_obj).request();
  } catch (const py::error_already_set&) {
    type_error("psi must be a 1-dimensional NumPy array");
  } catch (const std::exception&) {
    type_error("psi must be a 1-dimensional NumPy array");
  }
  if (info.ndim != 1) value_error("psi must be 1-dimensional");
  const bool c64 = info.format == "Zf" && info.itemsize == 8;
  const bool c128 = info.format == "Zd" && info.itemsize == 16;
  if (!c64 && !c128) type_error("psi dtype must be complex64 or complex128");
  if (info.shape[0] > 1 && info.strides[0] != info.itemsize) type_error("psi must be C-contiguous");
  const std::size_t n = static_cast<std::size_t>(info.shape[0]);
  return translate([&]() -> py::object {
    if (c128)
      return py::cast(op.expectation_statevector_complex128(
          std::span<const std::complex<double>>(static_cast<const std::complex<double>*>(info.ptr), n)));
    return py::cast(op.expectation_statevector_complex64(
        std::span<const std::complex<float>>(static_cast<const std::complex<float>*>(info.ptr), n)));
  });
}

struct CaiView {
  std::uintptr_t ptr = 0;
  DeviceStatevectorDtype dtype = DeviceStatevectorDtype::Complex128;
  std::size_t length = 0;
};

// __cuda_array_interface__ statevector (pauli_sum_py.cpp:438-502).
CaiView parse_cai(const py::handle& obj) {
  py::object iface = obj.attr("__cuda_array_interface__");
  if (!PyMapping_Check(iface.ptr())) type_error("__cuda_array_interface__ must be a mapping");
  py::dict d = py::reinterpret_borrow<py::dict>(iface);
  auto required = [&](const char* k) -> py::object {
    if (!d.contains(k)) type_error(std::string("__cuda_array_interface__ is missing required field ") + k);
    return d[k];
  };
  py::object shape = required("shape");
  if (!PySequence_Check(shape.ptr()) || PyUnicode_Check(shape.ptr()))
    type_error("__cuda_array_interface__ shape must be a sequence");
  if (PySequence_Size(shape.ptr()) != 1) value_error("CUDA statevector must be 1-dimensional");
  py::object s0 = py::reinterpret_borrow<py::sequence>(shape)[0];
  if (!PyLong_Check(s0.ptr())) type_error("shape must contain integers");
  const long long len = s0.cast<long long>();
  if (len < 0) value_error("CUDA statevector length must be non-negative");
  py::object ts = required("typestr");
  if (!PyUnicode_Check(ts.ptr())) type_error("__cuda_array_interface__ typestr must be a string");
  const std::string typestr = ts.cast<std::string>();
  CaiView v;
  std::size_t itemsize = 0;
  if (typestr == "<c16" || typestr == "=c16") {
    v.dtype = DeviceStatevectorDtype::Complex128;
    itemsize = 16;
  } else if (typestr == "<c8" || typestr == "=c8") {
    v.dtype = DeviceStatevectorDtype::Complex64;
    itemsize = 8;
  } else {
    type_error("CUDA statevector typestr must be native-endian complex64 or complex128");
  }
  if (d.contains("strides") && !d["strides"].is_none()) {
    py::object st = d["strides"];
    if (!PySequence_Check(st.ptr()) || PyUnicode_Check(st.ptr()) || PySequence_Size(st.ptr()) != 1)
      type_error("CUDA statevector strides must be None or a 1-item sequence");
    if (py::reinterpret_borrow<py::sequence>(st)[0].cast<long long>() != static_cast<long long>(itemsize))
      type_error("CUDA statevector must be C-contiguous");
  }
  py::object data = required("data");
  if (!PySequence_Check(data.ptr()) || PyUnicode_Check(data.ptr()) || PySequence_Size(data.ptr()) < 1)
    type_error("__cuda_array_interface__ data must be a sequence containing a pointer");
  py::object p = py::reinterpret_borrow<py::sequence>(data)[0];
  if (!PyLong_Check(p.ptr())) type_error("__cuda_array_interface__ data pointer must be an integer");
  const unsigned long long ptr = PyLong_AsUnsignedLongLong(p.ptr());
  if (PyErr_Occurred()) {
    PyErr_Clear();
    value_error("__cuda_array_interface__ data pointer is out of range");
  }
  if (ptr == 0 && len > 0) type_error("__cuda_array_interface__ data pointer must be non-null");
  v.ptr = ptr;
  v.length = static_cast<std::size_t>(len);
  return v;
}

py::dict device_dict(const CudaDeviceInfo& d) {
  py::dict out;
  out["ordinal"] = d.ordinal;
  out["name"] = d.name;
  out["compute_capability"] = py::make_tuple(d.compute_capability_major, d.compute_capability_minor);
  out["total_memory_bytes"] = d.total_memory_bytes;
  return out;
}

py::dict cuda_status_dict() {
  const CudaStatus s = DevicePauliSum::cuda_status();
  py::dict out;
  out["built"] = s.built;
  out["runtime_available"] = s.runtime_available;
  out["device_count"] = s.device_count;
  out["skip_reason"] = s.skip_reason;
  out["runtime_version"] = s.runtime_version;
  out["driver_version"] = s.driver_version;
  py::list devs;
  for (const auto& d : s.devices) devs.append(device_dict(d));
  out["devices"] = devs;
  return out;
}

AcceleratorBackend backend_arg(const py::object& b) {
  if (b.is_none()) return AcceleratorBackend::None;
  if (!PyUnicode_Check(b.ptr())) value_error("backend must be None, 'auto', 'cuda', 'hip', or 'metal'");
  return translate([&] { return accelerator_backend_from_name(b.cast<std::string>()); });
}

py::object axis_counts(const std::vector<std::uint64_t>& v) { return u64_array(v); }

// ------------------------------------------------------------- DLPack export
// DeviceCommutationMatrix.__dlpack__ keeps the reference's contract
// (bindings/python/pauli_sum_py.cpp:663-821, .pyi:29-30): a versioned,
// read-only capsule "dltensor_versioned" of the dense (rows, cols) uint8
// buffer, compact row-major; the consumer's max_version must be at least
// (1, 0) (a legacy capsule cannot carry the read-only flag) and the producer
// answers with the lower of it and the version it was built against;
// copy=True and stream=0 are refused.  The capsule holds a reference to the
// Python matrix object, so the buffer lives as long as any view of it.  The
// buffer is complete when exported (every call that writes it synchronises),
// so no stream ordering is needed: a stream token is only validated.

[[noreturn]] void buffer_error(const std::string& m) {
  PyErr_SetString(PyExc_BufferError, m.c_str());
  throw py::error_already_set();
}

struct MatrixDlpackContext {
  std::unique_ptr<std::int64_t[]> shape;
  std::unique_ptr<std::int64_t[]> strides;
  PyObject* owner = nullptr;  // strong reference to the exporting matrix
};

void matrix_dlpack_deleter(DLManagedTensorVersioned* managed) {
  if (managed == nullptr) return;
  auto* ctx = static_cast<MatrixDlpackContext*>(managed->manager_ctx);
  if (ctx != nullptr) {
    if (ctx->owner != nullptr) {
      PyGILState_STATE st = PyGILState_Ensure();  // consumers may call the deleter without the GIL
      Py_DECREF(ctx->owner);
      PyGILState_Release(st);
    }
    delete ctx;
  }
  delete managed;
}

// A capsule that no consumer took ("used_dltensor_versioned" once consumed)
// frees its tensor when it is collected.
void matrix_dlpack_capsule_destructor(PyObject* capsule) {
  if (PyCapsule_IsValid(capsule, "used_dltensor_versioned")) return;
  if (!PyCapsule_IsValid(capsule, "dltensor_versioned")) {
    PyErr_Clear();
    return;
  }
  auto* managed = static_cast<DLManagedTensorVersioned*>(PyCapsule_GetPointer(capsule, "dltensor_versioned"));
  if (managed != nullptr && managed->deleter != nullptr) managed->deleter(managed);
  else PyErr_Clear();
}

py::object matrix_dlpack(py::object self, py::object stream, py::object max_version, py::object copy,
                         py::object dl_device) {
  const auto& mtx = self.cast<const DeviceCommutationMatrix&>();
  // dl_device (DLPack >= 2023.12 consumers): only the matrix's own device
  if (!dl_device.is_none()) {
    py::tuple own = py::make_tuple(mtx.dlpack_device_type(), mtx.device());
    if (!dl_device.equal(own)) buffer_error("DeviceCommutationMatrix.__dlpack__ exports only on its own device");
  }
  if (!copy.is_none()) {
    const int truth = PyObject_IsTrue(copy.ptr());
    if (truth == 1) buffer_error("DeviceCommutationMatrix.__dlpack__ does not support copy=True");
    PyErr_Clear();
  }
  if (!stream.is_none()) {
    if (!PyLong_Check(stream.ptr())) type_error("stream must be None or an integer accelerator stream token");
    const long long token = stream.cast<long long>();
    if (token == 0) value_error("stream=0 is ambiguous in the Python DLPack protocol");
    if (token < 0) value_error("stream must be non-negative");
  }
  // consumer's highest version; None leaves no read-only capable version
  std::uint32_t major = 0, minor = 0;
  if (!max_version.is_none()) {
    if (!PyTuple_Check(max_version.ptr()) || PyTuple_Size(max_version.ptr()) != 2)
      value_error("max_version must be None or a (major, minor) tuple");
    py::tuple t = py::reinterpret_borrow<py::tuple>(max_version);
    long long a = 0, b = 0;
    try {
      a = t[0].cast<long long>();
      b = t[1].cast<long long>();
    } catch (const py::cast_error&) {
      value_error("max_version must be None or a (major, minor) tuple");
    }
    if (a < 0 || b < 0 || a > std::numeric_limits<std::uint32_t>::max() ||
        b > std::numeric_limits<std::uint32_t>::max())
      value_error("max_version components must be non-negative uint32 values");
    major = static_cast<std::uint32_t>(a);
    minor = static_cast<std::uint32_t>(b);
  }
  if (max_version.is_none() || major < 1)
    buffer_error("DeviceCommutationMatrix.__dlpack__ requires max_version >= (1, 0) "
                 "so the read-only DLPack contract can be represented");
  DLPackVersion version{DLPACK_MAJOR_VERSION, DLPACK_MINOR_VERSION};
  if (major < version.major || (major == version.major && minor < version.minor)) version = {major, minor};

  auto ctx = std::make_unique<MatrixDlpackContext>();
  ctx->shape = std::make_unique<std::int64_t[]>(2);
  ctx->strides = std::make_unique<std::int64_t[]>(2);
  ctx->shape[0] = static_cast<std::int64_t>(mtx.rows());
  ctx->shape[1] = static_cast<std::int64_t>(mtx.cols());
  ctx->strides[0] = static_cast<std::int64_t>(mtx.cols());
  ctx->strides[1] = 1;
  auto managed = std::make_unique<DLManagedTensorVersioned>();
  managed->version = version;
  managed->manager_ctx = ctx.get();
  managed->deleter = &matrix_dlpack_deleter;
  managed->flags = DLPACK_FLAG_BITMASK_READ_ONLY;
  managed->dl_tensor.data = reinterpret_cast<void*>(mtx.data_pointer_for_dlpack());
  managed->dl_tensor.device = DLDevice{static_cast<DLDeviceType>(mtx.dlpack_device_type()), mtx.device()};
  managed->dl_tensor.ndim = 2;
  managed->dl_tensor.dtype = DLDataType{static_cast<std::uint8_t>(kDLUInt), 8, 1};
  managed->dl_tensor.shape = ctx->shape.get();
  managed->dl_tensor.strides = ctx->strides.get();
  managed->dl_tensor.byte_offset = 0;
  PyObject* capsule = PyCapsule_New(managed.get(), "dltensor_versioned", &matrix_dlpack_capsule_destructor);
  if (capsule == nullptr) throw py::error_already_set();
  ctx->owner = self.ptr();
  Py_INCREF(ctx->owner);
  ctx.release();
  managed.release();
  return py::reinterpret_steal<py::object>(capsule);
}

}  // namespace

// PauliSum from packed words (numpy arrays, converted to the storage types).
PauliSum from_packed(long long n, py::array_t<std::uint64_t, py::array::c_style | py::array::forcecast> x,
                     py::array_t<std::uint64_t, py::array::c_style | py::array::forcecast> z,
                     py::array_t<std::complex<double>, py::array::c_style | py::array::forcecast> c) {
  std::vector<std::uint64_t> vx(x.data(), x.data() + x.size()), vz(z.data(), z.data() + z.size());
  std::vector<std::complex<double>> vc(c.data(), c.data() + c.size());
  return translate([&] {
    return PauliSum::from_packed(nonneg(n, "num_qubits"), std::move(vx), std::move(vz), std::move(vc));
  });
}

// (x, z, coeffs) copies of a PauliSum's storage as numpy arrays.
py::tuple to_packed(const PauliSum& p) {
  const auto T = static_cast<py::ssize_t>(p.num_terms());
  const auto W = static_cast<py::ssize_t>(p.words());
  py::array_t<std::uint64_t> x({T, W}), z({T, W});
  if (T * W) {
    std::memcpy(x.mutable_data(), p.x_words().data(), T * W * 8);
    std::memcpy(z.mutable_data(), p.z_words().data(), T * W * 8);
  }
  return py::make_tuple(x, z, coeff_array(p.coeffs()));
}

PYBIND11_MODULE(_wolfgang_core, m) {
  m.doc() = "B200 (sm_100a) packed-Pauli kernels behind the wolfgang_quantum API";

  py::class_<DeviceCommutationMatrix>(m, "DeviceCommutationMatrix",
                                      "Owning device-resident dense uint8 commutation matrix.")
      .def_static(
          "empty",
          [](py::handle shape, int device, py::object backend) {
            if (!PySequence_Check(shape.ptr()) || PyUnicode_Check(shape.ptr()))
              value_error("shape must be a 2-item sequence of non-negative integers");
            if (PySequence_Size(shape.ptr()) != 2) value_error("shape must contain exactly 2 dimensions");
            py::sequence s = py::reinterpret_borrow<py::sequence>(shape);
            const std::size_t rows = size_arg(s[0], "shape");
            const std::size_t cols = size_arg(s[1], "shape");
            return translate([&] { return DeviceCommutationMatrix::empty(rows, cols, backend_arg(backend), device); });
          },
          py::arg("shape"), py::arg("device") = 0, py::arg("backend") = py::none())
      .def_property_readonly("shape", [](const DeviceCommutationMatrix& mtx) { return py::make_tuple(mtx.rows(), mtx.cols()); })
      .def_property_readonly("device", &DeviceCommutationMatrix::device)
      .def_property_readonly("backend", &DeviceCommutationMatrix::backend)
      .def_property_readonly("dtype", [](const DeviceCommutationMatrix&) { return "uint8"; })
      .def_property_readonly("num_entries", &DeviceCommutationMatrix::num_entries)
      .def("to_host",
           [](const DeviceCommutationMatrix& mtx) {
             py::array a = bool_array(mtx.to_host());
             return a.reshape({static_cast<py::ssize_t>(mtx.rows()), static_cast<py::ssize_t>(mtx.cols())});
           })
      .def(
          "count_commuting",
          [](const DeviceCommutationMatrix& mtx, py::object axis) -> py::object {
            if (axis.is_none()) return py::int_(mtx.count_commuting());
            if (!PyLong_Check(axis.ptr())) value_error("axis must be None, 0, or 1");
            const long long a = axis.cast<long long>();
            if (a == 0) return axis_counts(mtx.count_commuting_cols());
            if (a == 1) return axis_counts(mtx.count_commuting_rows());
            value_error("axis must be None, 0, or 1");
          },
          py::arg("axis") = py::none())
      .def(
          "conflict_degrees",
          [](const DeviceCommutationMatrix& mtx, py::object axis) -> py::object {
            if (axis.is_none()) return py::int_(mtx.num_entries() - mtx.count_commuting());
            if (!PyLong_Check(axis.ptr())) value_error("axis must be None, 0, or 1");
            const long long a = axis.cast<long long>();
            if (a == 0) {
              auto v = mtx.count_commuting_cols();
              for (auto& x : v) x = mtx.rows() - x;
              return axis_counts(v);
            }
            if (a == 1) {
              auto v = mtx.count_commuting_rows();
              for (auto& x : v) x = mtx.cols() - x;
              return axis_counts(v);
            }
            value_error("axis must be None, 0, or 1");
          },
          py::arg("axis") = py::none())
      .def("__dlpack__", &matrix_dlpack, py::arg("stream") = py::none(), py::arg("max_version") = py::none(),
           py::arg("copy") = py::none(), py::arg("dl_device") = py::none(),
           "Read-only DLPack capsule of the dense (rows, cols) uint8 device buffer (DLPack >= 1.0).")
      .def("__dlpack_device__",
           [](const DeviceCommutationMatrix& mtx) { return py::make_tuple(mtx.dlpack_device_type(), mtx.device()); })
      .def_property_readonly("__cuda_array_interface__", [](const DeviceCommutationMatrix& mtx) {
        py::dict d;
        d["shape"] = py::make_tuple(mtx.rows(), mtx.cols());
        d["typestr"] = "|u1";
        d["data"] = py::make_tuple(mtx.data_pointer_for_cuda_array_interface(), true);
        d["version"] = 3;
        d["strides"] = py::none();
        return d;
      });

  py::class_<DeviceCommutationBits>(m, "DeviceCommutationBits",
                                    "Bit-packed device commutation matrix (uint32 words, row-major).")
      .def_property_readonly("shape", [](const DeviceCommutationBits& b) { return py::make_tuple(b.rows(), b.cols()); })
      .def_property_readonly("pitch_words", &DeviceCommutationBits::pitch_words)
      .def_property_readonly("device", &DeviceCommutationBits::device)
      .def_property_readonly("data_pointer", &DeviceCommutationBits::data_pointer)
      .def("to_host",
           [](const DeviceCommutationBits& b) {
             const auto v = b.to_host();
             py::array_t<std::uint32_t> a({static_cast<py::ssize_t>(b.rows()), static_cast<py::ssize_t>(b.pitch_words())});
             if (!v.empty()) std::memcpy(a.mutable_data(), v.data(), v.size() * 4);
             return a;
           })
      .def(
          "count_commuting",
          [](const DeviceCommutationBits& b, py::object axis) -> py::object {
            if (axis.is_none()) return py::int_(b.count_commuting());
            const long long a = axis.cast<long long>();
            if (a == 0) return axis_counts(b.count_commuting_cols());
            if (a == 1) return axis_counts(b.count_commuting_rows());
            value_error("axis must be None, 0, or 1");
          },
          py::arg("axis") = py::none());

  py::class_<DevicePauliSum>(m, "DevicePauliSum",
                             "Owning device mirror of a PauliSum. Construct with PauliSum.to_device().")
      .def_property_readonly("num_qubits", &DevicePauliSum::num_qubits)
      .def_property_readonly("num_terms", &DevicePauliSum::num_terms)
      .def_property_readonly("device", &DevicePauliSum::device)
      .def_property_readonly("backend", &DevicePauliSum::backend)
      .def_property_readonly("_pointers", [](const DevicePauliSum& d) {
        return py::make_tuple(d.x_pointer(), d.z_pointer(), d.coeffs_pointer());
      })
      .def("to_host", &DevicePauliSum::to_host)
      .def(
          "simplify", [](const DevicePauliSum& op, double atol, double rtol) { return translate([&] { return op.simplify(atol, rtol); }); },
          py::arg("atol") = 1.0e-12, py::arg("rtol") = 0.0)
      .def(
          "expectation_statevector",
          [](const DevicePauliSum& op, py::handle psi) -> py::object {
            if (py::hasattr(psi, "__cuda_array_interface__")) {
              const CaiView v = parse_cai(psi);
              return translate([&] { return py::cast(op.expectation_statevector_device_pointer(v.ptr, v.dtype, v.length)); });
            }
            return host_expectation(op, psi);
          },
          py::arg("psi"))
      .def(
          "commutes_with",
          [](const DevicePauliSum& l, const DevicePauliSum& r, py::handle max_entries) -> py::object {
            const std::size_t me = size_arg(max_entries, "max_commutation_matrix_entries");
            return translate([&] { return shape_flags(l.commutes_with(r, me), l.num_terms(), r.num_terms()); });
          },
          py::arg("other"), py::arg("max_commutation_matrix_entries") = 100000000)
      .def(
          "commutes_with_into",
          [](const DevicePauliSum& l, const DevicePauliSum& r, py::handle output, py::handle max_entries) {
            const std::size_t me = size_arg(max_entries, "max_commutation_matrix_entries");
            translate([&] {
              (void)PauliSum::checked_commutation_matrix_entries_for_testing(l.num_terms(), r.num_terms(), me);
              return 0;
            });
            py::buffer_info info = py::reinterpret_borrow<py::buffer>(output).request(true);
            if (!(info.format == "?" && info.itemsize == 1)) type_error("commutes_with_into output dtype must be bool");
            if (info.ndim != 1) value_error("commutes_with_into output must be a 1-dimensional array");
            if (info.shape[0] > 1 && info.strides[0] != 1) type_error("commutes_with_into output must be C-contiguous");
            translate([&] {
              l.commutes_with_into(r, std::span<std::uint8_t>(static_cast<std::uint8_t*>(info.ptr),
                                                              static_cast<std::size_t>(info.shape[0])),
                                   me);
              return 0;
            });
          },
          py::arg("other"), py::arg("output"), py::arg("max_commutation_matrix_entries") = 100000000)
      .def(
          "commutes_with_device",
          [](const DevicePauliSum& l, const DevicePauliSum& r, py::handle max_entries, py::object output) -> py::object {
            const std::size_t me = size_arg(max_entries, "max_commutation_matrix_entries");
            if (output.is_none()) return translate([&] { return py::cast(l.commutes_with_device(r, me)); });
            if (!py::isinstance<DeviceCommutationMatrix>(output))
              type_error("commutes_with_device output must be a DeviceCommutationMatrix");
            auto& out = output.cast<DeviceCommutationMatrix&>();
            translate([&] {
              l.commutes_with_device_into(r, out, me);
              return 0;
            });
            return output;
          },
          py::arg("other"), py::arg("max_commutation_matrix_entries") = 100000000, py::arg("output") = py::none())
      .def(
          "commutes_with_bits",
          [](const DevicePauliSum& l, const DevicePauliSum& r, py::handle max_entries, int algo) {
            const std::size_t me = size_arg(max_entries, "max_entries");
            return translate([&] { return l.commutes_with_bits(r, me, algo); });
          },
          py::arg("other"), py::arg("max_entries") = (1ull << 40), py::arg("algo") = 0)
      .def(
          "matmul",
          [](const DevicePauliSum& l, const DevicePauliSum& r, bool simplify, py::handle max_terms) {
            const std::size_t mt = size_arg(max_terms, "max_intermediate_terms");
            return translate([&] { return l.matmul(r, simplify, mt); });
          },
          py::arg("rhs"), py::arg("simplify") = true, py::arg("max_intermediate_terms") = 50000000)
      .def(
          "group_commuting",
          [](const DevicePauliSum& op, std::string mode, std::string strategy) {
            return translate([&] { return op.group_commuting(mode, strategy); });
          },
          py::arg("mode") = "qwc", py::arg("strategy") = "largest_first");

  py::class_<PauliSum>(m, "PauliSum",
                       "Sparse sum of Pauli strings backed by packed x/z bit masks and complex128 coefficients.")
      .def(py::init([](long long n, long long t) { return PauliSum(nonneg(n, "num_qubits"), nonneg(t, "num_terms")); }),
           py::arg("num_qubits"), py::arg("num_terms") = 0)
      .def_static("empty", [](long long n) { return PauliSum::empty(nonneg(n, "num_qubits")); }, py::arg("num_qubits"))
      .def_static(
          "from_labels",
          [](py::handle labels, py::object coeffs) {
            auto l = parse_labels(labels);
            auto c = parse_coeffs(coeffs, l.size());
            return translate([&] { return PauliSum::from_labels(l, c); });
          },
          py::arg("labels"), py::arg("coeffs") = py::none())
      .def_static(
          "from_sparse_list",
          [](py::handle triples, long long n) {
            auto t = parse_sparse(triples);
            return translate([&] { return PauliSum::from_sparse_list(t, nonneg(n, "num_qubits")); });
          },
          py::arg("triples"), py::arg("num_qubits"))
      .def_static("from_packed", from_packed, py::arg("num_qubits"), py::arg("x"), py::arg("z"), py::arg("coeffs"),
                  "Build from packed words: x/z uint64 (num_terms, words), bit q of word q // 64 for qubit q;\n"
                  "coeffs complex128 (num_terms,).  No labels are parsed; unused high bits of the last\n"
                  "word must be zero.  (An addition: the reference builds only from labels or sparse lists.)")
      .def_static("_from_packed", from_packed, py::arg("num_qubits"), py::arg("x"), py::arg("z"), py::arg("coeffs"))
      .def("to_packed", to_packed,
           "The packed words and coefficients: (x, z) uint64 arrays (num_terms, words) and a complex128\n"
           "array (num_terms,), copies of the storage.")
      .def("_packed", to_packed)
      .def_property_readonly("num_qubits", &PauliSum::num_qubits)
      .def_property_readonly("num_terms", &PauliSum::num_terms)
      .def(
          "to_device",
          [](const PauliSum& op, int device, py::object backend) {
            return translate([&] { return DevicePauliSum::from_host(op, backend_arg(backend), device); });
          },
          py::arg("device") = 0, py::arg("backend") = py::none())
      .def("to_labels",
           [](const PauliSum& op) {
             py::list labels;
             for (const auto& l : op.to_labels()) labels.append(l);
             return py::make_tuple(labels, coeff_array(op.coeffs()));
           })
      .def("to_sparse_list",
           [](const PauliSum& op) {
             py::list out;
             for (const auto& t : op.to_sparse_list()) {
               py::list idx;
               for (auto q : t.qubit_indices) idx.append(q);
               out.append(py::make_tuple(t.local_pauli_string, idx, t.coefficient));
             }
             return out;
           })
      .def(
          "simplify", [](const PauliSum& op, double atol, double rtol) { return translate([&] { return op.simplify(atol, rtol); }); },
          py::arg("atol") = 1.0e-12, py::arg("rtol") = 0.0)
      .def("__add__", [](const PauliSum& a, const PauliSum& b) { return translate([&] { return a.add(b); }); }, py::is_operator())
      .def("__mul__", [](const PauliSum& a, py::handle s) { return a.scalar_multiply(complex_arg(s, "scalar")); }, py::is_operator())
      .def("__rmul__", [](const PauliSum& a, py::handle s) { return a.scalar_multiply(complex_arg(s, "scalar")); }, py::is_operator())
      .def(
          "matmul",
          [](const PauliSum& l, const PauliSum& r, bool simplify, py::handle max_terms) {
            const std::size_t mt = size_arg(max_terms, "max_intermediate_terms");
            return translate([&] { return l.matmul(r, simplify, mt); });
          },
          py::arg("rhs"), py::arg("simplify") = true, py::arg("max_intermediate_terms") = 50000000)
      .def("__matmul__", [](const PauliSum& l, const PauliSum& r) { return translate([&] { return l.matmul(r); }); },
           py::is_operator())
      .def(
          "commutes_with",
          [](const PauliSum& l, const PauliSum& r, py::handle max_entries) -> py::object {
            const std::size_t me = size_arg(max_entries, "max_commutation_matrix_entries");
            return translate([&] { return shape_flags(l.commutes_with(r, me), l.num_terms(), r.num_terms()); });
          },
          py::arg("other"), py::arg("max_commutation_matrix_entries") = 100000000)
      .def(
          "group_commuting",
          [](const PauliSum& op, std::string mode, std::string strategy, py::handle max_terms) {
            const std::size_t mt = size_arg(max_terms, "max_terms_for_graph");
            return translate([&] { return op.group_commuting(mode, strategy, mt); });
          },
          py::arg("mode") = "qwc", py::arg("strategy") = "largest_first", py::arg("max_terms_for_graph") = 50000)
      .def("expectation_statevector", [](const PauliSum& op, py::handle psi) { return host_expectation(op, psi); },
           py::arg("psi"))
      .def(
          "expectation_z_counts",
          [](const PauliSum& op, py::handle counts) {
            if (!PyMapping_Check(counts.ptr())) value_error("counts must be a mapping from dense bitstrings to numeric counts");
            std::vector<std::string> bits;
            std::vector<double> vals;
            py::object items = counts.attr("items")();
            for (py::handle item : py::iter(items)) {
              py::tuple kv = py::reinterpret_borrow<py::tuple>(item);
              if (!PyUnicode_Check(kv[0].ptr())) value_error("Z-count bitstrings must be strings");
              bits.push_back(kv[0].cast<std::string>());
              const double v = PyFloat_AsDouble(kv[1].ptr());
              if (PyErr_Occurred()) {
                PyErr_Clear();
                value_error("Z-count values must be numeric");
              }
              vals.push_back(v);
            }
            return translate([&] { return op.expectation_z_counts(bits, vals); });
          },
          py::arg("counts"))
      .def_static(
          "_checked_commutation_size_for_testing",
          [](py::handle l, py::handle r, py::handle me) {
            return translate([&] {
              return PauliSum::checked_commutation_matrix_entries_for_testing(
                  size_arg(l, "lhs_terms"), size_arg(r, "rhs_terms"), size_arg(me, "max_commutation_matrix_entries"));
            });
          },
          py::arg("lhs_terms"), py::arg("rhs_terms"), py::arg("max_commutation_matrix_entries"))
      .def_static(
          "_checked_matmul_size_for_testing",
          [](py::handle l, py::handle r, py::handle mt) {
            return translate([&] {
              return PauliSum::checked_matmul_intermediate_terms_for_testing(
                  size_arg(l, "lhs_terms"), size_arg(r, "rhs_terms"), size_arg(mt, "max_intermediate_terms"));
            });
          },
          py::arg("lhs_terms"), py::arg("rhs_terms"), py::arg("max_intermediate_terms"));

  m.def("cuda_available", &DevicePauliSum::cuda_available);
  m.def("cuda_devices", []() {
    py::list out;
    for (const auto& d : DevicePauliSum::cuda_status().devices) out.append(device_dict(d));
    return out;
  });
  m.def("hip_available", []() { return false; });
  m.def("hip_devices", []() { return py::list(); });
  m.def("metal_available", []() { return false; });
  m.def("metal_devices", []() { return py::list(); });
  m.def("_cuda_status", &cuda_status_dict);
  m.def("_build_info", []() {
    py::dict d;
    d["version"] = "0.2.3+b200";
    d["cuda_architectures"] = "100a";
    d["compiled_backends"] = py::make_tuple("cuda");
    d["abi_version"] = wg_abi_version();
    d["cuda"] = cuda_status_dict();
    return d;
  });
}
