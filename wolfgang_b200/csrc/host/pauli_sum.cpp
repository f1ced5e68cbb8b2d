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
#include <cmath>
#include <complex>
#include <condition_variable>
#include <cstring>
#include <deque>
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
// that the download then overwrites, and filling one by appending is a single
// copy stream.  Here, per vector, the storage is reserved and advised for
// transparent huge pages, and three stages run over slices of the download's
// chunk size, each slice after the previous stage has finished it:
//   fault -- a pool of threads pre-faults the slices (MADV_POPULATE_WRITE), in
//            download order across the three vectors;
//   size  -- one thread per vector grows the vector over the faulted slice
//            (resize: a zero fill of pages already present);
//   copy  -- the downloaded chunk (x, z and the coefficients are downloaded
//            concurrently, each through its own pinned staging) is copied
//            into the sized slice by several threads of a copy pool.
// Each thread writes distinct elements, and the vector object itself is only
// touched by its sizing thread; the storage never moves (the capacity is
// reserved first).  Small results take the plain path.
constexpr std::size_t kBigHostBytes = std::size_t{64} << 20;
constexpr std::size_t kSliceBytes = std::size_t{64} << 20;  // = the chunk size of wg_memcpy_dtoh_chunked

// Done flags of one stage over a vector's slices.
struct SliceFlags {
  std::unique_ptr<std::atomic<bool>[]> done;
  std::mutex mu;
  std::condition_variable cv;
  void init(std::size_t n) {
    done.reset(new std::atomic<bool>[n]);
    for (std::size_t k = 0; k < n; ++k) done[k].store(false, std::memory_order_relaxed);
  }
  void mark(std::size_t k) {
    {
      std::lock_guard<std::mutex> lk(mu);
      done[k].store(true, std::memory_order_release);
    }
    cv.notify_all();
  }
  void wait(std::size_t k) {
    if (done[k].load(std::memory_order_acquire)) return;
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return done[k].load(std::memory_order_acquire); });
  }
};

// Slices [k * kSliceBytes, (k + 1) * kSliceBytes) of one vector's storage.
struct FaultPlan {
  char* base = nullptr;
  std::size_t bytes = 0;
  SliceFlags faulted, sized;
  std::size_t slices() const { return (bytes + kSliceBytes - 1) / kSliceBytes; }
  void init(void* p, std::size_t n) {
    base = static_cast<char*>(p);
    bytes = n;
    faulted.init(slices());
    sized.init(slices());
#ifdef MADV_HUGEPAGE
    const std::size_t page = static_cast<std::size_t>(sysconf(_SC_PAGESIZE));
    const std::uintptr_t lo = (reinterpret_cast<std::uintptr_t>(p) + page - 1) & ~(page - 1);
    const std::uintptr_t hi = (reinterpret_cast<std::uintptr_t>(p) + n) & ~(page - 1);
    if (hi > lo) madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_HUGEPAGE);  // advice only
#endif
  }
  // Faults in the whole pages inside slice k (pages shared with a neighbour
  // are faulted by the first write), then marks it.
  void fault(std::size_t k) {
#ifdef MADV_POPULATE_WRITE
    const std::size_t page = static_cast<std::size_t>(sysconf(_SC_PAGESIZE));
    const std::uintptr_t a = reinterpret_cast<std::uintptr_t>(base) + k * kSliceBytes;
    const std::uintptr_t e = reinterpret_cast<std::uintptr_t>(base) + std::min(bytes, (k + 1) * kSliceBytes);
    const std::uintptr_t lo = (a + page - 1) & ~(page - 1), hi = e & ~(page - 1);
    if (hi > lo) madvise(reinterpret_cast<void*>(lo), hi - lo, MADV_POPULATE_WRITE);
#endif
    faulted.mark(k);
  }
};

// Worker threads that copy pieces of chunks; a copy call returns once all of
// its pieces are done.  Without workers the caller copies alone.
class CopyPool {
 public:
  explicit CopyPool(unsigned n) {
    try {
      for (unsigned t = 0; t < n; ++t) workers_.emplace_back([this] { work(); });
    } catch (const std::system_error&) {  // fewer workers
    }
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void copy(void* dst, const void* src, std::size_t bytes) {
    constexpr std::size_t kPiece = std::size_t{8} << 20;
    const std::size_t pieces = (bytes + kPiece - 1) / kPiece;
    if (workers_.empty() || pieces < 2) {
      std::memcpy(dst, src, bytes);
      return;
    }
    Done done;
    done.left = pieces - 1;
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (std::size_t q = 1; q < pieces; ++q)
        tasks_.push_back(Task{static_cast<char*>(dst) + q * kPiece, static_cast<const char*>(src) + q * kPiece,
                              std::min(kPiece, bytes - q * kPiece), &done});
    }
    cv_.notify_all();
    std::memcpy(dst, src, std::min(kPiece, bytes));  // the first piece, here
    std::unique_lock<std::mutex> lk(done.mu);
    done.cv.wait(lk, [&] { return done.left == 0; });
  }

 private:
  struct Done {
    std::mutex mu;
    std::condition_variable cv;
    std::size_t left = 0;
  };
  struct Task {
    char* dst;
    const char* src;
    std::size_t bytes;
    Done* done;
  };
  void work() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || !tasks_.empty(); });
        if (tasks_.empty()) return;
        t = tasks_.front();
        tasks_.pop_front();
      }
      std::memcpy(t.dst, t.src, t.bytes);
      {
        std::lock_guard<std::mutex> lk(t.done->mu);
        --t.done->left;
      }
      t.done->cv.notify_all();
    }
  }
  std::vector<std::thread> workers_;
  std::deque<Task> tasks_;
  std::mutex mu_;
  std::condition_variable cv_;
  bool stop_ = false;
};

// Grows v (capacity reserved) to `count` elements, one faulted slice at a time.
template <typename T>
void size_by_slices(std::vector<T>& v, std::size_t count, FaultPlan& plan) {
  const std::size_t per = kSliceBytes / sizeof(T);
  for (std::size_t k = 0; k < plan.slices(); ++k) {
    plan.faulted.wait(k);
    v.resize(std::min(count, (k + 1) * per));
    plan.sized.mark(k);
  }
}

// Downloads the device buffer's first `count` elements into base (the reserved
// storage of a vector being sized by size_by_slices): chunk k is copied once
// slice k is sized.
template <typename T>
void download_into_slices(const DeviceBuffer& b, T* base, std::size_t count, FaultPlan& plan, CopyPool& pool) {
  struct Ctx {
    char* base;
    FaultPlan* plan;
    CopyPool* pool;
    std::size_t k;
  } ctx{reinterpret_cast<char*>(base), &plan, &pool, 0};
  auto fn = [](void* user, const void* chunk, std::size_t bytes) {
    auto* c = static_cast<Ctx*>(user);
    const std::size_t k = c->k++;
    c->plan->sized.wait(k);
    c->pool->copy(c->base + k * kSliceBytes, chunk, bytes);
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
  x.reserve(words_total);
  z.reserve(words_total);
  c.reserve(terms);
  FaultPlan plans[3];
  plans[0].init(x.data(), 8 * words_total);
  plans[1].init(z.data(), 8 * words_total);
  plans[2].init(c.data(), 16 * terms);
  // the storage, taken before any thread resizes a vector (it never moves)
  std::uint64_t* const xs = x.data();
  std::uint64_t* const zs = z.data();
  std::complex<double>* const cs = c.data();
  const unsigned hw = std::max(4u, std::min(32u, std::thread::hardware_concurrency()));
  CopyPool pool(hw > 6 ? hw - 6 : 1);  // besides the three download and three sizing threads
  // fault work in download order: slice 0 of x, z, c, then slice 1, ...
  std::atomic<std::size_t> next{0};
  const std::size_t most = std::max(plans[0].slices(), plans[2].slices());
  auto faulter = [&] {
    for (std::size_t w; (w = next.fetch_add(1)) < 3 * most;) {
      FaultPlan& pl = plans[w % 3];
      if (w / 3 < pl.slices()) pl.fault(w / 3);
    }
  };
  std::vector<std::thread> faulters;
  try {
    for (unsigned t = 0; t + 3 < hw; ++t) faulters.emplace_back(faulter);
  } catch (const std::system_error&) {  // no threads to spare: the faulting runs here, first
  }
  if (faulters.empty()) faulter();
  std::thread sx([&] { size_by_slices(x, words_total, plans[0]); });
  std::thread sz([&] { size_by_slices(z, words_total, plans[1]); });
  std::thread sc([&] { size_by_slices(c, terms, plans[2]); });
  std::exception_ptr ex, ez, ec;
  std::thread tx([&] {
    try {
      download_into_slices(bx, xs, words_total, plans[0], pool);
    } catch (...) {
      ex = std::current_exception();
    }
  });
  std::thread tz([&] {
    try {
      download_into_slices(bz, zs, words_total, plans[1], pool);
    } catch (...) {
      ez = std::current_exception();
    }
  });
  try {
    download_into_slices(bc, cs, terms, plans[2], pool);
  } catch (...) {
    ec = std::current_exception();
  }
  tx.join();
  tz.join();
  // every slice is faulted and sized whatever the downloads did, so these end
  sx.join();
  sz.join();
  sc.join();
  for (auto& t : faulters) t.join();
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
