// PauliSum host implementation.
//
// Storage, parsing, export and the O(T) arithmetic follow the reference's host
// semantics (src/pauli_sum.cpp:14-43, src/parse.cpp:15-97, src/export.cpp:12-53,
// src/arithmetic.cpp:14-57) with the same error messages.  Every compute method
// uploads its operands and runs on the GPU through the wg_* C-ABI.

#include "wolfgang/pauli_sum.hpp"

#include <algorithm>
#include <atomic>
#include <bit>
#include <chrono>
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <unordered_set>
#include <utility>
#include <vector>

#include <sys/mman.h>
#include <unistd.h>

#include "abi.hpp"
#include "guards.hpp"

namespace wolfgang {

using abi::DeviceBuffer;

namespace {

bool valid_pauli(char p) { return p == 'I' || p == 'X' || p == 'Y' || p == 'Z'; }

void set_bit(std::vector<std::uint64_t>& v, std::size_t words, std::size_t term, std::size_t q) {
  v[term * words + q / 64] |= std::uint64_t{1} << (q % 64);
}

char letter(bool xb, bool zb) { return xb ? (zb ? 'Y' : 'X') : (zb ? 'Z' : 'I'); }

// Result vectors of a large download.  A value-initialised std::vector of
// many gigabytes spends its construction on page faults and on writing zeros
// that the download then overwrites.  Here each vector's storage is reserved
// and advised for transparent huge pages, and the vector grows by appending
// the downloaded chunks (x, z and the coefficients download concurrently,
// each through its own pinned staging, and each download thread appends to
// its own vector).  The appends go piece by piece over a grid of 2 MiB
// aligned pieces, and helper threads fault in (MADV_POPULATE_WRITE) the
// pieces a short distance ahead of the append: the kernel's zero fill of a
// page and the append's stores then meet the same lines while they are still
// in the caches, instead of each writing the page to memory.  The vector
// object is only touched by its download thread; the helpers touch pages of
// the reserved storage, which never moves.  Small results take the plain path.
constexpr std::size_t kBigHostBytes = std::size_t{64} << 20;
constexpr std::size_t kPieceBytes = std::size_t{2} << 20;
constexpr std::size_t kFaultAhead = 2;  // pieces a helper may fault beyond the append

// Faults in the pieces of [base, base + bytes) ahead of an append.
class FaultAhead {
 public:
  FaultAhead(void* base, std::size_t bytes, unsigned threads)
      : base_(reinterpret_cast<std::uintptr_t>(base)),
        bytes_(bytes),
        grid_(base_ & ~std::uintptr_t{kPieceBytes - 1}),
        pieces_((base_ + bytes - grid_ + kPieceBytes - 1) / kPieceBytes),
        faulted_(new bool[pieces_]()) {
#ifdef MADV_HUGEPAGE
    const std::uintptr_t lo = round_up(base_), hi = round_down(base_ + bytes_);
    if (hi > lo) madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_HUGEPAGE);  // advice only
#endif
#ifdef MADV_POPULATE_WRITE
    try {
      for (unsigned t = 0; t < threads; ++t) helpers_.emplace_back([this] { work(); });
    } catch (const std::system_error&) {  // fewer helpers: the appends fault what is left
    }
#else
    (void)threads;
#endif
  }
  ~FaultAhead() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : helpers_) t.join();
  }
  FaultAhead(const FaultAhead&) = delete;
  FaultAhead& operator=(const FaultAhead&) = delete;

  // Byte offsets from base where piece k starts and ends (base is 16-byte
  // aligned, so every piece holds whole elements).
  std::size_t start(std::size_t k) const { return k == 0 ? 0 : grid_ + k * kPieceBytes - base_; }
  std::size_t end(std::size_t k) const { return k + 1 < pieces_ ? start(k + 1) : bytes_; }
  std::size_t piece_of(std::size_t off) const { return (base_ + off - grid_) / kPieceBytes; }

  // Waits until piece k is faulted in (at once when no helper runs).
  void wait(std::size_t k) {
    if (helpers_.empty()) return;
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return faulted_[k]; });
  }
  // The append has filled pieces [0, k]: helpers may fault up to k + 1 + kFaultAhead.
  void appended(std::size_t k) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      appended_ = k + 1;
    }
    cv_.notify_all();
  }

 private:
  static std::uintptr_t page() { return static_cast<std::uintptr_t>(sysconf(_SC_PAGESIZE)); }
  static std::uintptr_t round_up(std::uintptr_t a) { return (a + page() - 1) & ~(page() - 1); }
  static std::uintptr_t round_down(std::uintptr_t a) { return a & ~(page() - 1); }
  void work() {
    for (;;) {
      const std::size_t k = next_.fetch_add(1);
      if (k >= pieces_) return;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || k <= appended_ + kFaultAhead; });
        if (stop_) return;
      }
#ifdef MADV_POPULATE_WRITE
      // whole pages inside the piece; a page shared with a neighbour piece
      // (only at the ends of the storage) is faulted by the first write
      const std::uintptr_t lo = round_up(base_ + start(k)), hi = round_down(base_ + end(k));
      if (hi > lo) madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_POPULATE_WRITE);
#endif
      {
        std::lock_guard<std::mutex> lk(mu_);
        faulted_[k] = true;
      }
      cv_.notify_all();
    }
  }
  const std::uintptr_t base_;
  const std::size_t bytes_;
  const std::uintptr_t grid_;  // base rounded down to the piece grid
  const std::size_t pieces_;
  std::unique_ptr<bool[]> faulted_;
  std::size_t appended_ = 0;  // pieces [0, appended_) are filled
  std::atomic<std::size_t> next_{0};
  bool stop_ = false;
  std::mutex mu_;
  std::condition_variable cv_;
  std::vector<std::thread> helpers_;
};

// Downloads the device buffer's first `count` elements and appends them to v
// (capacity reserved, empty), piece by piece behind the fault-ahead helpers.
template <typename T>
void download_appending(const DeviceBuffer& b, std::vector<T>& v, std::size_t count, FaultAhead& ahead) {
  struct Ctx {
    std::vector<T>* v;
    FaultAhead* ahead;
    std::size_t off;  // bytes appended so far
  } ctx{&v, &ahead, 0};
  auto fn = [](void* user, const void* chunk, std::size_t bytes) {
    auto* c = static_cast<Ctx*>(user);
    const char* src = static_cast<const char*>(chunk);
    for (std::size_t done = 0; done < bytes;) {
      const std::size_t k = c->ahead->piece_of(c->off);
      const std::size_t n = std::min(bytes - done, c->ahead->end(k) - c->off);
      c->ahead->wait(k);
      const T* s = reinterpret_cast<const T*>(src + done);
      c->v->insert(c->v->end(), s, s + n / sizeof(T));
      done += n;
      c->off += n;
      if (c->off == c->ahead->end(k)) c->ahead->appended(k);
    }
  };
  abi::check(wg_memcpy_dtoh_chunked(b.device(), b.get(), count * sizeof(T), fn, &ctx, nullptr));
}

void fetch_result_vectors(const DeviceBuffer& bx, const DeviceBuffer& bz, const DeviceBuffer& bc,
                          std::size_t words_total, std::size_t terms, std::vector<std::uint64_t>& x,
                          std::vector<std::uint64_t>& z, std::vector<std::complex<double>>& c) {
  if (16 * words_total + 16 * terms < kBigHostBytes) {
    x.resize(words_total);
    z.resize(words_total);
    c.resize(terms);
    bx.download(x.data(), x.size() * 8);
    bz.download(z.data(), z.size() * 8);
    bc.download(c.data(), c.size() * 16);
    return;
  }
  // WG_HOST_TRACE set: when each vector is filled, on stderr
  const bool trace = std::getenv("WG_HOST_TRACE") != nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  auto ms = [&] { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };
  double t_filled[3] = {0.0, 0.0, 0.0};
  x.clear();
  z.clear();
  c.clear();
  x.reserve(words_total);
  z.reserve(words_total);
  c.reserve(terms);
  auto aligned16 = [](const void* p) { return reinterpret_cast<std::uintptr_t>(p) % 16 == 0; };
  if (!aligned16(x.data()) || !aligned16(z.data()) || !aligned16(c.data())) {  // not from this allocator
    x.resize(words_total);
    z.resize(words_total);
    c.resize(terms);
    bx.download(x.data(), x.size() * 8);
    bz.download(z.data(), z.size() * 8);
    bc.download(c.data(), c.size() * 16);
    return;
  }
  // two helpers per vector where the host has the threads (a helper faults at
  // about half the rate an append consumes pages)
  const unsigned helpers = std::thread::hardware_concurrency() >= 9 ? 2 : 1;
  FaultAhead ax(x.data(), 8 * words_total, helpers);
  FaultAhead az(z.data(), 8 * words_total, helpers);
  FaultAhead ac(c.data(), 16 * terms, helpers);
  std::exception_ptr ex, ez, ec;
  std::thread tx([&] {
    try {
      download_appending(bx, x, words_total, ax);
      t_filled[0] = ms();
    } catch (...) {
      ex = std::current_exception();
    }
  });
  std::thread tz([&] {
    try {
      download_appending(bz, z, words_total, az);
      t_filled[1] = ms();
    } catch (...) {
      ez = std::current_exception();
    }
  });
  try {
    download_appending(bc, c, terms, ac);
    t_filled[2] = ms();
  } catch (...) {
    ec = std::current_exception();
  }
  tx.join();
  tz.join();
  if (trace)
    std::fprintf(stderr, "host result %.2f GB: x %.1f ms, z %.1f ms, coefficients %.1f ms\n",
                 (16.0 * words_total + 16.0 * terms) * 1e-9, t_filled[0], t_filled[1], t_filled[2]);
  for (const auto& e : {ex, ez, ec})
    if (e) std::rethrow_exception(e);
}

// Operands of one compute call, resident on the compute device.
struct DeviceOperand {
  DeviceBuffer x, z, c;
};

DeviceOperand upload(int device, const PauliSum& p) {
  DeviceOperand d;
  const std::size_t packed = p.num_terms() * p.words();
  d.x = abi::upload_vector(device, p.x_words().data(), packed);
  d.z = abi::upload_vector(device, p.z_words().data(), packed);
  d.c = abi::upload_vector(device, p.coeffs().data(), p.num_terms());
  return d;
}

// Sampled duplicate rate of the first min(T, 512) keys; the reference takes
// its fused hash-accumulate matmul path when an operand with >= 128 terms has
// >= 25 % duplicates there (src/multiply.cpp:29-69, :107-109, :179-181).
bool duplicate_heavy(const PauliSum& p) {
  if (p.num_terms() < 128) return false;
  const std::size_t s = std::min<std::size_t>(p.num_terms(), 512);
  const std::size_t w = p.words();
  std::vector<std::vector<std::uint64_t>> keys(s);
  for (std::size_t t = 0; t < s; ++t)
    for (std::size_t k = 0; k < w; ++k) {
      keys[t].push_back(p.x_words()[t * w + k]);
      keys[t].push_back(p.z_words()[t * w + k]);
    }
  std::sort(keys.begin(), keys.end());
  const std::size_t unique = static_cast<std::size_t>(std::unique(keys.begin(), keys.end()) - keys.begin());
  return 1.0 - static_cast<double>(unique) / static_cast<double>(s) >= 0.25;
}

}  // namespace

// ------------------------------------------------------------------ storage

PauliSum::PauliSum(std::size_t num_qubits, std::size_t num_terms)
    : num_qubits_(num_qubits),
      words_(guards::word_count(num_qubits)),
      num_terms_(num_terms),
      x_(guards::product(num_terms, words_, "x"), 0),
      z_(guards::product(num_terms, words_, "z"), 0),
      coeffs_(num_terms, std::complex<double>{0.0, 0.0}) {}

PauliSum::PauliSum(std::size_t num_qubits, std::size_t words, std::size_t num_terms, std::vector<std::uint64_t> x,
                   std::vector<std::uint64_t> z, std::vector<std::complex<double>> coeffs)
    : num_qubits_(num_qubits),
      words_(words),
      num_terms_(num_terms),
      x_(std::move(x)),
      z_(std::move(z)),
      coeffs_(std::move(coeffs)) {
  const std::size_t packed = guards::product(num_terms_, words_, "packed");
  if (x_.size() != packed || z_.size() != packed || coeffs_.size() != num_terms_)
    throw std::invalid_argument("PauliSum buffer sizes do not match metadata");
}

PauliSum PauliSum::empty(std::size_t num_qubits) {
  return PauliSum(num_qubits, guards::word_count(num_qubits), 0, {}, {}, {});
}

PauliSum PauliSum::from_packed(std::size_t num_qubits, std::vector<std::uint64_t> x, std::vector<std::uint64_t> z,
                               std::vector<std::complex<double>> coeffs) {
  const std::size_t words = guards::word_count(num_qubits);
  const std::size_t T = coeffs.size();
  if (x.size() != T * words || z.size() != T * words)
    throw std::invalid_argument("PauliSum buffer sizes do not match metadata");
  if (words && num_qubits % 64) {
    const std::uint64_t high = ~((std::uint64_t{1} << (num_qubits % 64)) - 1);
    for (std::size_t t = 0; t < T; ++t)
      if ((x[t * words + words - 1] | z[t * words + words - 1]) & high)
        throw std::invalid_argument("packed Pauli words set bits above num_qubits");
  }
  return PauliSum(num_qubits, words, T, std::move(x), std::move(z), std::move(coeffs));
}

std::size_t PauliSum::num_qubits() const noexcept { return num_qubits_; }
std::size_t PauliSum::num_terms() const noexcept { return num_terms_; }
std::size_t PauliSum::words() const noexcept { return words_; }
const std::vector<std::uint64_t>& PauliSum::x_words() const noexcept { return x_; }
const std::vector<std::uint64_t>& PauliSum::z_words() const noexcept { return z_; }
const std::vector<std::complex<double>>& PauliSum::coeffs() const noexcept { return coeffs_; }

// ------------------------------------------------------------------ I/O

PauliSum PauliSum::from_labels(const std::vector<std::string>& labels,
                               const std::vector<std::complex<double>>& coeffs) {
  if (labels.empty())
    throw std::invalid_argument(
        "PauliSum.from_labels([]) cannot infer num_qubits; use PauliSum.empty(num_qubits)");
  if (coeffs.size() != labels.size()) throw std::invalid_argument("coefficient count must match label count");
  const std::size_t n = labels.front().size();
  const std::size_t words = guards::word_count(n);
  const std::size_t T = labels.size();
  std::vector<std::uint64_t> x(guards::product(T, words, "x"), 0), z(guards::product(T, words, "z"), 0);
  for (std::size_t t = 0; t < T; ++t) {
    const std::string& label = labels[t];
    if (label.size() != n) throw std::invalid_argument("all dense labels must have the same length");
    for (std::size_t i = 0; i < n; ++i) {
      const char p = label[i];
      if (!valid_pauli(p)) throw std::invalid_argument("dense labels may contain only I, X, Y, or Z");
      const std::size_t q = n - 1 - i;  // right-most character is qubit 0
      if (p == 'X' || p == 'Y') set_bit(x, words, t, q);
      if (p == 'Z' || p == 'Y') set_bit(z, words, t, q);
    }
  }
  return PauliSum(n, words, T, std::move(x), std::move(z), coeffs);
}

PauliSum PauliSum::from_sparse_list(const std::vector<SparseTerm>& terms, std::size_t num_qubits) {
  const std::size_t words = guards::word_count(num_qubits);
  const std::size_t T = terms.size();
  std::vector<std::uint64_t> x(guards::product(T, words, "x"), 0), z(guards::product(T, words, "z"), 0);
  std::vector<std::complex<double>> coeffs;
  coeffs.reserve(T);
  for (std::size_t t = 0; t < T; ++t) {
    const SparseTerm& s = terms[t];
    if (s.local_pauli_string.size() != s.qubit_indices.size())
      throw std::invalid_argument("sparse local_pauli_string length must match qubit_indices length");
    std::unordered_set<std::size_t> seen;
    for (std::size_t i = 0; i < s.local_pauli_string.size(); ++i) {
      const char p = s.local_pauli_string[i];
      if (!valid_pauli(p)) throw std::invalid_argument("sparse local_pauli_string may contain only I, X, Y, or Z");
      const std::size_t q = s.qubit_indices[i];
      if (q >= num_qubits) throw std::invalid_argument("sparse qubit index is out of range");
      if (!seen.insert(q).second) throw std::invalid_argument("sparse term contains a duplicate qubit index");
      if (p == 'X' || p == 'Y') set_bit(x, words, t, q);
      if (p == 'Z' || p == 'Y') set_bit(z, words, t, q);
    }
    coeffs.push_back(s.coefficient);
  }
  return PauliSum(num_qubits, words, T, std::move(x), std::move(z), std::move(coeffs));
}

std::vector<std::string> PauliSum::to_labels() const {
  std::vector<std::string> out;
  out.reserve(num_terms_);
  for (std::size_t t = 0; t < num_terms_; ++t) {
    std::string label(num_qubits_, 'I');
    for (std::size_t q = 0; q < num_qubits_; ++q) {
      const std::uint64_t bit = std::uint64_t{1} << (q % 64);
      const std::size_t w = t * words_ + q / 64;
      label[num_qubits_ - 1 - q] = letter(x_[w] & bit, z_[w] & bit);
    }
    out.push_back(std::move(label));
  }
  return out;
}

std::vector<PauliSum::SparseTerm> PauliSum::to_sparse_list() const {
  std::vector<SparseTerm> out;
  out.reserve(num_terms_);
  for (std::size_t t = 0; t < num_terms_; ++t) {
    SparseTerm s;
    s.coefficient = coeffs_[t];
    for (std::size_t q = 0; q < num_qubits_; ++q) {
      const std::uint64_t bit = std::uint64_t{1} << (q % 64);
      const std::size_t w = t * words_ + q / 64;
      const char p = letter(x_[w] & bit, z_[w] & bit);
      if (p != 'I') {
        s.local_pauli_string.push_back(p);
        s.qubit_indices.push_back(q);
      }
    }
    out.push_back(std::move(s));
  }
  return out;
}

// ------------------------------------------------------------------ arithmetic

PauliSum PauliSum::add(const PauliSum& rhs) const {
  if (num_qubits_ != rhs.num_qubits_) throw std::invalid_argument("PauliSum addition requires the same num_qubits");
  const std::size_t T = guards::sum(num_terms_, rhs.num_terms_, "terms");
  std::vector<std::uint64_t> x, z;
  std::vector<std::complex<double>> c;
  x.reserve(guards::product(T, words_, "x"));
  z.reserve(guards::product(T, words_, "z"));
  c.reserve(T);
  x.insert(x.end(), x_.begin(), x_.end());
  x.insert(x.end(), rhs.x_.begin(), rhs.x_.end());
  z.insert(z.end(), z_.begin(), z_.end());
  z.insert(z.end(), rhs.z_.begin(), rhs.z_.end());
  c.insert(c.end(), coeffs_.begin(), coeffs_.end());
  c.insert(c.end(), rhs.coeffs_.begin(), rhs.coeffs_.end());
  return PauliSum(num_qubits_, words_, T, std::move(x), std::move(z), std::move(c));
}

PauliSum PauliSum::scalar_multiply(std::complex<double> scalar) const {
  std::vector<std::complex<double>> c;
  c.reserve(coeffs_.size());
  for (const auto& v : coeffs_) c.push_back(v * scalar);
  return PauliSum(num_qubits_, words_, num_terms_, x_, z_, std::move(c));
}

// ------------------------------------------------------------------ device compute

PauliSum PauliSum::download_device_result(std::size_t n, std::size_t words, int device, std::uint64_t* ox,
                                          std::uint64_t* oz, double* oc, std::size_t U) {
  DeviceBuffer bx = DeviceBuffer::adopt(device, ox, U * words * 8);
  DeviceBuffer bz = DeviceBuffer::adopt(device, oz, U * words * 8);
  DeviceBuffer bc = DeviceBuffer::adopt(device, oc, U * 16);
  if (U == 0) return PauliSum::empty(n);
  std::vector<std::uint64_t> x, z;
  std::vector<std::complex<double>> c;
  fetch_result_vectors(bx, bz, bc, U * words, U, x, z, c);
  return PauliSum(n, words, U, std::move(x), std::move(z), std::move(c));
}

PauliSum PauliSum::simplify(double atol, double rtol) const {
  if (atol < 0.0 || rtol < 0.0 || !std::isfinite(atol) || !std::isfinite(rtol))
    throw std::invalid_argument("simplify tolerances must be non-negative finite values");
  if (num_terms_ == 0) return PauliSum::empty(num_qubits_);
  const int dev = abi::compute_device();
  DeviceOperand d = upload(dev, *this);
  std::uint64_t *ox = nullptr, *oz = nullptr;
  double* oc = nullptr;
  std::size_t U = 0;
  abi::check(wg_simplify(dev, words_, num_terms_, d.x.as<std::uint64_t>(), d.z.as<std::uint64_t>(),
                         d.c.as<double>(), atol, rtol, &ox, &oz, &oc, &U, nullptr));
  return download_device_result(num_qubits_, words_, dev, ox, oz, oc, U);
}

PauliSum PauliSum::matmul(const PauliSum& rhs, bool simplify_output, std::size_t max_intermediate_terms) const {
  if (num_qubits_ != rhs.num_qubits_) throw std::invalid_argument("PauliSum matmul requires the same num_qubits");
  const std::size_t P = guards::matmul_terms(num_terms_, rhs.num_terms_, max_intermediate_terms);
  if (P == 0) return PauliSum::empty(num_qubits_);
  int mode = WG_PRODUCTS_RAW;
  if (simplify_output) {
    const bool fused = (words_ == 1 || words_ == 2) && (duplicate_heavy(*this) || duplicate_heavy(rhs));
    mode = fused ? WG_PRODUCTS_FUSED : WG_PRODUCTS_SIMPLIFY;
  }
  const int dev = abi::compute_device();
  DeviceOperand l = upload(dev, *this), r = upload(dev, rhs);
  std::uint64_t *ox = nullptr, *oz = nullptr;
  double* oc = nullptr;
  std::size_t U = 0;
  abi::check(wg_pauli_products(dev, words_, l.x.as<std::uint64_t>(), l.z.as<std::uint64_t>(), l.c.as<double>(),
                               num_terms_, r.x.as<std::uint64_t>(), r.z.as<std::uint64_t>(), r.c.as<double>(),
                               rhs.num_terms_, mode, 1.0e-12, 0.0, &ox, &oz, &oc, &U, nullptr));
  if (!simplify_output) {
    // raw products keep nested-loop order and are returned as-is
    DeviceBuffer bx = DeviceBuffer::adopt(dev, ox, U * words_ * 8);
    DeviceBuffer bz = DeviceBuffer::adopt(dev, oz, U * words_ * 8);
    DeviceBuffer bc = DeviceBuffer::adopt(dev, oc, U * 16);
    std::vector<std::uint64_t> x, z;
    std::vector<std::complex<double>> c;
    fetch_result_vectors(bx, bz, bc, U * words_, U, x, z, c);
    return PauliSum(num_qubits_, words_, U, std::move(x), std::move(z), std::move(c));
  }
  return download_device_result(num_qubits_, words_, dev, ox, oz, oc, U);
}

std::vector<std::uint8_t> PauliSum::commutes_with(const PauliSum& rhs,
                                                  std::size_t max_commutation_matrix_entries) const {
  if (num_qubits_ != rhs.num_qubits_)
    throw std::invalid_argument("PauliSum commutation requires the same num_qubits");
  const std::size_t entries = guards::commutation_entries(num_terms_, rhs.num_terms_, max_commutation_matrix_entries);
  std::vector<std::uint8_t> out(entries, 0);
  if (entries == 0) return out;
  const int dev = abi::compute_device();
  DeviceOperand l = upload(dev, *this), r = upload(dev, rhs);
  const std::size_t pitch = (rhs.num_terms_ + 31) / 32;
  DeviceBuffer bits(dev, num_terms_ * pitch * 4), flags(dev, entries);
  const int algo = abi::commutation_algo_for(words_, x_.data(), z_.data(), num_terms_, rhs.num_terms_);
  abi::check(wg_commutation_bits(dev, words_, l.x.as<std::uint64_t>(), l.z.as<std::uint64_t>(), num_terms_,
                                 r.x.as<std::uint64_t>(), r.z.as<std::uint64_t>(), rhs.num_terms_,
                                 bits.as<std::uint32_t>(), pitch, algo, nullptr));
  abi::check(wg_bits_to_u8(dev, bits.as<std::uint32_t>(), num_terms_, rhs.num_terms_, pitch,
                           flags.as<std::uint8_t>(), nullptr));
  flags.download(out.data(), entries);
  return out;
}

std::vector<PauliSum> PauliSum::group_commuting(std::string_view mode, std::string_view strategy,
                                                std::size_t max_terms_for_graph) const {
  // max_terms_for_graph only chooses between the reference's precomputed-graph
  // and streaming checks, which give identical groups (src/grouping.cpp:137-193).
  (void)max_terms_for_graph;
  if (strategy != "largest_first") throw std::invalid_argument("group_commuting strategy must be 'largest_first'");
  if (mode != "qwc" && mode != "full") throw std::invalid_argument("group_commuting mode must be 'qwc' or 'full'");
  if (num_terms_ == 0) return {};
  const int dev = abi::compute_device();
  DeviceOperand d = upload(dev, *this);
  std::vector<std::size_t> order(num_terms_), sizes(num_terms_);
  std::size_t G = 0;
  abi::check(wg_group_commuting(dev, words_, num_terms_, d.x.as<std::uint64_t>(), d.z.as<std::uint64_t>(),
                                mode == "full" ? 1 : 0, order.data(), sizes.data(), &G, nullptr));
  std::vector<PauliSum> groups;
  groups.reserve(G);
  std::size_t p = 0;
  for (std::size_t g = 0; g < G; ++g) {
    std::vector<std::uint64_t> x, z;
    std::vector<std::complex<double>> c;
    for (std::size_t i = 0; i < sizes[g]; ++i, ++p) {
      const std::size_t t = order[p];
      for (std::size_t k = 0; k < words_; ++k) {
        x.push_back(x_[t * words_ + k]);
        z.push_back(z_[t * words_ + k]);
      }
      c.push_back(coeffs_[t]);
    }
    groups.push_back(PauliSum(num_qubits_, words_, sizes[g], std::move(x), std::move(z), std::move(c)));
  }
  return groups;
}

namespace {

template <typename C>
std::complex<double> expectation_on_device(const PauliSum& op, std::span<const C> psi, int dtype) {
  guards::statevector_length(op.num_qubits(), psi.size());
  if (op.num_terms() == 0) return {0.0, 0.0};
  const int dev = abi::compute_device();
  DeviceOperand d = upload(dev, op);
  DeviceBuffer dpsi = abi::upload_vector(dev, psi.data(), psi.size());
  double out[2] = {0.0, 0.0};
  abi::check(wg_expectation(dev, op.num_qubits(), op.num_terms(), d.x.as<std::uint64_t>(), d.z.as<std::uint64_t>(),
                            d.c.as<double>(), dpsi.get(), dtype, out, nullptr));
  return {out[0], out[1]};
}

}  // namespace

std::complex<double> PauliSum::expectation_statevector_complex128(std::span<const std::complex<double>> psi) const {
  return expectation_on_device(*this, psi, WG_DTYPE_C128);
}

std::complex<double> PauliSum::expectation_statevector_complex64(std::span<const std::complex<float>> psi) const {
  return expectation_on_device(*this, psi, WG_DTYPE_C64);
}

std::complex<double> PauliSum::expectation_z_counts(const std::vector<std::string>& bitstrings,
                                                    const std::vector<double>& counts) const {
  // Validation order and messages of src/expectation.cpp:157-230.
  if (bitstrings.size() != counts.size())
    throw std::invalid_argument("Z-count bitstring and count arrays must have the same length");
  for (std::uint64_t w : x_)
    if (w != 0) throw std::invalid_argument("expectation_z_counts requires diagonal Pauli terms");
  double total = 0.0;
  for (double v : counts) {
    if (v < 0.0) throw std::invalid_argument("Z-count values must be non-negative");
    if (!std::isfinite(v)) throw std::invalid_argument("Z-count values must be finite");
    total += v;
  }
  if (total <= 0.0) throw std::invalid_argument("Z-count total count must be positive");
  const std::size_t rows = bitstrings.size();
  std::vector<std::uint64_t> packed(guards::product(rows, words_, "counts"), 0);
  for (std::size_t r = 0; r < rows; ++r) {
    const std::string& b = bitstrings[r];
    if (b.size() != num_qubits_) throw std::invalid_argument("Z-count bitstring length must equal num_qubits");
    for (std::size_t i = 0; i < b.size(); ++i) {
      if (b[i] != '0' && b[i] != '1') throw std::invalid_argument("Z-count bitstrings may contain only 0 or 1");
      if (b[i] == '1') {
        const std::size_t q = num_qubits_ - 1 - i;
        packed[r * words_ + q / 64] |= std::uint64_t{1} << (q % 64);
      }
    }
  }
  if (num_terms_ == 0) return {0.0, 0.0};
  const int dev = abi::compute_device();
  DeviceOperand d = upload(dev, *this);
  DeviceBuffer dp = abi::upload_vector(dev, packed.data(), packed.size());
  DeviceBuffer dc = abi::upload_vector(dev, counts.data(), counts.size());
  double out[2] = {0.0, 0.0};
  abi::check(wg_expectation_z_counts(dev, words_, num_terms_, d.x.as<std::uint64_t>(), d.z.as<std::uint64_t>(),
                                     d.c.as<double>(), rows, dp.as<std::uint64_t>(), dc.as<double>(), out, nullptr));
  return {out[0], out[1]};
}

std::size_t PauliSum::checked_matmul_intermediate_terms_for_testing(std::size_t lhs_terms, std::size_t rhs_terms,
                                                                     std::size_t max_intermediate_terms) {
  return guards::matmul_terms(lhs_terms, rhs_terms, max_intermediate_terms);
}

std::size_t PauliSum::checked_commutation_matrix_entries_for_testing(std::size_t lhs_terms, std::size_t rhs_terms,
                                                                      std::size_t max_commutation_matrix_entries) {
  return guards::commutation_entries(lhs_terms, rhs_terms, max_commutation_matrix_entries);
}

}  // namespace wolfgang
