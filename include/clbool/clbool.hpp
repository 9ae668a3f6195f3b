// clbool.hpp -- C++ host layer of the B200 back end, mirroring the
// reference's public surface (include/clbool.hpp) over the C ABI in
// clbool_b200.h.  Header-only; link against libclbool_b200.so.
//
//   Controls, create_controls, show_devices   src/core/controls.hpp, src/common/env.hpp
//   Status, Exception                          src/core/error.hpp:130-213
//   matrix_dcsr / matrix_coo / matrix_csr      src/core/matrix_{dcsr,coo,csr}.hpp
//   matrix_*_cpu                               src/core/cpu_matrices.hpp
//   dcsr::, coo::, csr:: operations            src/dcsr/dcsr.hpp, src/coo/coo.hpp, src/csr/csr.hpp
//   conversions                                src/common/matrices_conversions.hpp
//   prefix_sum, fill_with                      src/common/cl_operations.hpp
//
// Device arrays are held by shared_ptr, so copies of matrices are shallow
// (the reference's cl::Buffer is reference counted the same way) and
// conversions documented as "shallow for cols" share the column array.
// Row pointers are uint64 on the device (the reference uses uint32).
#pragma once

#include <clbool_b200.h>

#include <cstdint>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <utility>
#include <sstream>
#include <string>
#include <vector>

namespace clbool {

enum Status {
    CLBOOL_NO_SUCH_PROGRAM,
    CLBOOL_CREATE_KERNEL_ERROR,
    CLBOOL_BUILD_PROGRAM_ERROR,
    CLBOOL_INCOMPLETE_KERNEL,
    CLBOOL_RUN_KERNEL_FAILURE,
    CLBOOL_EVENT_WAITING_ERROR,
    CLBOOL_CREATE_BUFFER_ERROR,
    CLBOOL_COPY_BUFFER_ERROR,
    CLBOOL_READ_BUFFER_ERROR,
    CLBOOL_WRITE_BUFFER_ERROR,
    CLBOOL_CREATE_CONTROLS_ERROR,
    CLBOOL_INVALID_ARGUMENT,
    CLBOOL_INVALID_VALUE,
    CLBOOL_INITIALIZATION_ERROR,
    CLBOOL_DEVICE_STATUS_ERROR,
    CLBOOL_NOT_SUPPORTED
};

class Exception : public std::exception {
    std::string message_;
    Status status_;

public:
    Exception(std::string message, Status status) : message_(std::move(message)), status_(status) {}
    const char *what() const noexcept override { return message_.c_str(); }
    Status status() const { return status_; }
    std::string get_message() const { return message_; }
};

namespace details {
inline Status to_status(int code) {
    if (code >= 1 && code <= 14) return static_cast<Status>(code - 1);
    if (code == CLB_DEVICE_STATUS_ERROR) return CLBOOL_DEVICE_STATUS_ERROR;
    if (code == CLB_NOT_SUPPORTED) return CLBOOL_NOT_SUPPORTED;
    return CLBOOL_RUN_KERNEL_FAILURE;
}
inline void check(int code) {
    if (code != CLB_SUCCESS) {
        std::string msg = std::string("[") + clb_status_string(code) + "] " + clb_last_error();
        throw Exception(msg, to_status(code));
    }
}
}  // namespace details

// ------------------------------------------------------------------ controls
struct Controls {
    std::shared_ptr<clb_controls> handle;
    int device = 0;

    explicit Controls(int device_id = 0) : device(device_id) {
        clb_controls *h = nullptr;
        details::check(clb_controls_create(device_id, &h));
        handle = std::shared_ptr<clb_controls>(h, [](clb_controls *p) { clb_controls_destroy(p); });
    }
    clb_controls *get() const { return handle.get(); }
    void sync() const { details::check(clb_controls_sync(get())); }
    // hands the memory pool's cached, unused device memory back (clb_controls_trim)
    void trim() const { details::check(clb_controls_trim(get())); }
};

inline Controls create_controls(uint32_t platform_id = 0, uint32_t device_id = 0) {
    if (platform_id != 0) throw Exception("no platform with id " + std::to_string(platform_id),
                                          CLBOOL_CREATE_CONTROLS_ERROR);
    return Controls(static_cast<int>(device_id));
}

inline void show_devices() {
    int n = 0;
    details::check(clb_device_count(&n));
    for (int d = 0; d < n; ++d) {
        char name[256];
        int sms = 0;
        uint64_t mem = 0;
        details::check(clb_device_info(d, name, sizeof(name), &sms, &mem));
        std::cout << "device id: " << d << "  " << name << "  SMs=" << sms << "  mem=" << (mem >> 20) << " MiB\n";
    }
}

// ------------------------------------------------------------ device memory
class Buffer {
    std::shared_ptr<void> ptr_;
    size_t bytes_ = 0;

public:
    Buffer() = default;
    // Takes ownership of a library allocation.
    Buffer(const Controls &c, void *p, size_t bytes) : bytes_(bytes) {
        auto h = c.handle;
        ptr_ = std::shared_ptr<void>(p, [h](void *q) {
            if (q) clb_free(h.get(), q);
        });
    }
    static Buffer create(const Controls &c, size_t bytes) {
        void *p = nullptr;
        details::check(clb_malloc(c.get(), bytes, &p));
        return Buffer(c, p, bytes);
    }
    template <class T>
    static Buffer upload(const Controls &c, const T *src, size_t n) {
        if (n == 0) return Buffer();
        Buffer b = create(c, n * sizeof(T));
        details::check(clb_memcpy_h2d(c.get(), b.get(), src, n * sizeof(T)));
        return b;
    }
    template <class T>
    std::vector<T> download(const Controls &c, size_t n) const {
        std::vector<T> out(n);
        if (n) details::check(clb_memcpy_d2h(c.get(), out.data(), get(), n * sizeof(T)));
        return out;
    }
    void *get() const { return ptr_.get(); }
    size_t bytes() const { return bytes_; }
    explicit operator bool() const { return ptr_ != nullptr; }
};

// -------------------------------------------------------------- host types
using cpu_buffer = std::vector<uint32_t>;
using coordinates = std::pair<uint32_t, uint32_t>;
using matrix_coo_cpu_pairs = std::vector<coordinates>;

struct matrix_dcsr_cpu {
    std::vector<uint64_t> rpt;
    cpu_buffer rows, cols;
};
struct matrix_coo_cpu {
    cpu_buffer rows, cols;
};
struct matrix_csr_cpu {
    std::vector<uint64_t> rpt;
    cpu_buffer cols;
    uint64_t nrows = 0, ncols = 0;
};

// ------------------------------------------------------------ device types
namespace details {
class matrix_base {
protected:
    uint64_t _nrows = 0, _ncols = 0, _nnz = 0;

public:
    using index_type = uint32_t;
    matrix_base() = default;
    matrix_base(uint64_t r, uint64_t c, uint64_t n) : _nrows(r), _ncols(c), _nnz(n) {}
    uint64_t nrows() const { return _nrows; }
    uint64_t ncols() const { return _ncols; }
    uint64_t nnz() const { return _nnz; }
    bool empty() const { return _nnz == 0; }
};
}  // namespace details

class matrix_dcsr : public details::matrix_base {
    Buffer _rpt, _rows, _cols;
    uint64_t _nzr = 0;

public:
    matrix_dcsr() = default;
    matrix_dcsr(uint64_t nrows, uint64_t ncols) : matrix_base(nrows, ncols, 0) {}
    matrix_dcsr(Buffer rpt, Buffer rows, Buffer cols, uint64_t nrows, uint64_t ncols, uint64_t nnz, uint64_t nzr)
        : matrix_base(nrows, ncols, nnz), _rpt(std::move(rpt)), _rows(std::move(rows)), _cols(std::move(cols)),
          _nzr(nzr) {}
    uint64_t nzr() const { return _nzr; }
    const Buffer &rpt_gpu() const { return _rpt; }
    const Buffer &rows_gpu() const { return _rows; }
    const Buffer &cols_gpu() const { return _cols; }
    clb_dcsr view() const {
        return clb_dcsr{_nrows, _ncols, _nnz, _nzr, (uint64_t *)_rpt.get(), (uint32_t *)_rows.get(),
                        (uint32_t *)_cols.get()};
    }
    // Wrap a clb_dcsr returned by the library; `cols_shared` keeps a column
    // array that the result shares with an input.
    static matrix_dcsr adopt(const Controls &c, const clb_dcsr &s, const Buffer *cols_shared = nullptr) {
        if (s.nnz == 0) return matrix_dcsr(s.nrows, s.ncols);
        Buffer cols = (cols_shared && cols_shared->get() == s.cols) ? *cols_shared : Buffer(c, s.cols, s.nnz * 4);
        return matrix_dcsr(Buffer(c, s.rpt, (s.nzr + 1) * 8), Buffer(c, s.rows, s.nzr * 4), cols, s.nrows, s.ncols,
                           s.nnz, s.nzr);
    }
};

class matrix_csr : public details::matrix_base {
    Buffer _rpt, _cols;

public:
    matrix_csr() = default;
    matrix_csr(uint64_t nrows, uint64_t ncols) : matrix_base(nrows, ncols, 0) {}
    matrix_csr(Buffer rpt, Buffer cols, uint64_t nrows, uint64_t ncols, uint64_t nnz)
        : matrix_base(nrows, ncols, nnz), _rpt(std::move(rpt)), _cols(std::move(cols)) {}
    const Buffer &rpt_gpu() const { return _rpt; }
    const Buffer &cols_gpu() const { return _cols; }
    clb_csr view() const { return clb_csr{_nrows, _ncols, _nnz, (uint64_t *)_rpt.get(), (uint32_t *)_cols.get()}; }
    static matrix_csr adopt(const Controls &c, const clb_csr &s, const Buffer *cols_shared = nullptr) {
        if (s.nnz == 0) return matrix_csr(s.nrows, s.ncols);
        Buffer cols = (cols_shared && cols_shared->get() == s.cols) ? *cols_shared : Buffer(c, s.cols, s.nnz * 4);
        return matrix_csr(Buffer(c, s.rpt, (s.nrows + 1) * 8), cols, s.nrows, s.ncols, s.nnz);
    }
};

class matrix_coo : public details::matrix_base {
    Buffer _rows, _cols;

public:
    matrix_coo() = default;
    matrix_coo(uint64_t nrows, uint64_t ncols) : matrix_base(nrows, ncols, 0) {}
    matrix_coo(Buffer rows, Buffer cols, uint64_t nrows, uint64_t ncols, uint64_t nnz)
        : matrix_base(nrows, ncols, nnz), _rows(std::move(rows)), _cols(std::move(cols)) {}
    // matrix_coo(controls, rows, cols, nrows, ncols, nnz, sorted, noDuplicates)
    // (src/core/matrix_coo.cpp:17-47).
    matrix_coo(const Controls &c, const uint32_t *rows, const uint32_t *cols, uint64_t nrows, uint64_t ncols,
               uint64_t nnz, bool sorted = true, bool noDuplicates = true)
        : matrix_base(nrows, ncols, nnz) {
        if (nnz == 0) return;
        _rows = Buffer::upload(c, rows, nnz);
        _cols = Buffer::upload(c, cols, nnz);
        if (!sorted) details::check(clb_coo_sort(c.get(), (uint32_t *)_rows.get(), (uint32_t *)_cols.get(), nnz));
        if (!noDuplicates) {
            clb_coo in = view(), out{};
            details::check(clb_coo_reduce_duplicates(c.get(), &in, &out));
            *this = adopt(c, out);
        }
    }
    const Buffer &rows_gpu() const { return _rows; }
    const Buffer &cols_gpu() const { return _cols; }
    clb_coo view() const { return clb_coo{_nrows, _ncols, _nnz, (uint32_t *)_rows.get(), (uint32_t *)_cols.get()}; }
    static matrix_coo adopt(const Controls &c, const clb_coo &s, const Buffer *rows_shared = nullptr,
                            const Buffer *cols_shared = nullptr) {
        if (s.nnz == 0) return matrix_coo(s.nrows, s.ncols);
        Buffer rows = (rows_shared && rows_shared->get() == s.rows) ? *rows_shared : Buffer(c, s.rows, s.nnz * 4);
        Buffer cols = (cols_shared && cols_shared->get() == s.cols) ? *cols_shared : Buffer(c, s.cols, s.nnz * 4);
        return matrix_coo(rows, cols, s.nrows, s.ncols, s.nnz);
    }
};

// ---------------------------------------------------------------- primitives
inline uint64_t prefix_sum(Controls &c, Buffer &array, uint64_t &total_sum, uint64_t array_size) {
    uint64_t t = 0;
    details::check(clb_prefix_sum_u32(c.get(), (uint32_t *)array.get(), array_size, &t));
    total_sum = t;
    return t;
}

inline void fill_with(Controls &c, Buffer &array, uint64_t size, uint32_t value) {
    details::check(clb_fill_u32(c.get(), (uint32_t *)array.get(), size, value));
}
inline void fill_with_zeroes(Controls &c, Buffer &array, uint64_t size) { fill_with(c, array, size, 0); }

// --------------------------------------------------------------- conversions
inline matrix_dcsr coo_to_dcsr_shallow(Controls &c, const matrix_coo &a) {
    if (a.empty()) return matrix_dcsr(a.nrows(), a.ncols());
    clb_coo in = a.view();
    clb_dcsr out{};
    details::check(clb_coo_to_dcsr(c.get(), &in, &out, 0));
    return matrix_dcsr::adopt(c, out, &a.cols_gpu());
}

inline matrix_coo dcsr_to_coo_shallow(Controls &c, const matrix_dcsr &a) {
    if (a.empty()) return matrix_coo(a.nrows(), a.ncols());
    clb_dcsr in = a.view();
    clb_coo out{};
    details::check(clb_dcsr_to_coo(c.get(), &in, &out, 0));
    return matrix_coo::adopt(c, out, nullptr, &a.cols_gpu());
}

inline matrix_coo dcsr_to_coo_deep(Controls &c, const matrix_dcsr &a) {
    if (a.empty()) return matrix_coo(a.nrows(), a.ncols());
    clb_dcsr in = a.view();
    clb_coo out{};
    details::check(clb_dcsr_to_coo(c.get(), &in, &out, 1));
    return matrix_coo::adopt(c, out);
}

// shallow for cols!
inline matrix_csr dcsr_to_csr(Controls &c, const matrix_dcsr &m) {
    if (m.empty()) return matrix_csr(m.nrows(), m.ncols());
    clb_dcsr in = m.view();
    clb_csr out{};
    details::check(clb_dcsr_to_csr(c.get(), &in, &out));
    return matrix_csr::adopt(c, out, &m.cols_gpu());
}

// shallow for cols!
inline matrix_dcsr csr_to_dcsr(Controls &c, const matrix_csr &m) {
    if (m.empty()) return matrix_dcsr(m.nrows(), m.ncols());
    clb_csr in = m.view();
    clb_dcsr out{};
    details::check(clb_csr_to_dcsr(c.get(), &in, &out));
    return matrix_dcsr::adopt(c, out, &m.cols_gpu());
}

inline matrix_dcsr matrix_dcsr_from_cpu(Controls &c, const matrix_dcsr_cpu &m, uint64_t size) {
    if (m.cols.empty()) return matrix_dcsr(size, size);
    return matrix_dcsr(Buffer::upload(c, m.rpt.data(), m.rpt.size()), Buffer::upload(c, m.rows.data(), m.rows.size()),
                       Buffer::upload(c, m.cols.data(), m.cols.size()), size, size, m.cols.size(), m.rows.size());
}

inline matrix_dcsr_cpu matrix_dcsr_from_gpu(Controls &c, const matrix_dcsr &m) {
    if (m.empty()) return {};
    return {m.rpt_gpu().download<uint64_t>(c, m.nzr() + 1), m.rows_gpu().download<uint32_t>(c, m.nzr()),
            m.cols_gpu().download<uint32_t>(c, m.nnz())};
}

inline matrix_coo_cpu matrix_coo_from_gpu(Controls &c, const matrix_coo &m) {
    if (m.empty()) return {};
    return {m.rows_gpu().download<uint32_t>(c, m.nnz()), m.cols_gpu().download<uint32_t>(c, m.nnz())};
}

inline matrix_csr_cpu matrix_csr_from_gpu(Controls &c, const matrix_csr &m) {
    if (m.empty()) return {{}, {}, m.nrows(), m.ncols()};
    return {m.rpt_gpu().download<uint64_t>(c, m.nrows() + 1), m.cols_gpu().download<uint32_t>(c, m.nnz()), m.nrows(),
            m.ncols()};
}

inline matrix_csr_cpu csr_cpu_from_pairs(const matrix_coo_cpu_pairs &mat, uint64_t m, uint64_t n) {
    matrix_csr_cpu out;
    out.nrows = m;
    out.ncols = n;
    out.rpt.assign(m + 1, 0);
    out.cols.resize(mat.size());
    for (size_t j = 0; j < mat.size(); ++j) {
        out.rpt[mat[j].first + 1]++;
        out.cols[j] = mat[j].second;
    }
    for (uint64_t i = 0; i < m; ++i) out.rpt[i + 1] += out.rpt[i];
    return out;
}

inline matrix_csr csr_from_cpu(Controls &c, const matrix_csr_cpu &m) {
    if (m.cols.empty()) return matrix_csr(m.nrows, m.ncols);
    return matrix_csr(Buffer::upload(c, m.rpt.data(), m.rpt.size()), Buffer::upload(c, m.cols.data(), m.cols.size()),
                      m.nrows, m.ncols, m.cols.size());
}

// ---------------------------------------------------------------- operations
namespace dcsr {
inline void matrix_multiplication_hash(Controls &c, matrix_dcsr &matrix_out, const matrix_dcsr &a,
                                       const matrix_dcsr &b, clb_spgemm_stats *stats = nullptr) {
    clb_dcsr va = a.view(), vb = b.view(), out{};
    details::check(clb_dcsr_spgemm_hash(c.get(), &va, &vb, &out, stats));
    matrix_out = matrix_dcsr::adopt(c, out);
}

inline void matrix_multiplication(Controls &c, matrix_dcsr &matrix_out, const matrix_dcsr &a, const matrix_dcsr &b,
                                  clb_spgemm_stats *stats = nullptr) {
    clb_dcsr va = a.view(), vb = b.view(), out{};
    details::check(clb_dcsr_spgemm_esc(c.get(), &va, &vb, &out, stats));
    matrix_out = matrix_dcsr::adopt(c, out);
}

inline void kronecker_product(Controls &c, matrix_dcsr &matrix_c, const matrix_dcsr &matrix_a,
                              const matrix_dcsr &matrix_b) {
    clb_dcsr va = matrix_a.view(), vb = matrix_b.view(), out{};
    details::check(clb_dcsr_kronecker(c.get(), &va, &vb, &out));
    matrix_c = matrix_dcsr::adopt(c, out);
}

inline void transpose(Controls &c, matrix_dcsr &matrix_out, const matrix_dcsr &matrix_in) {
    clb_dcsr v = matrix_in.view(), out{};
    details::check(clb_dcsr_transpose(c.get(), &v, &out));
    matrix_out = matrix_dcsr::adopt(c, out);
}

inline void submatrix(Controls &c, matrix_dcsr &matrix_out, const matrix_dcsr &matrix_in, uint32_t i, uint32_t j,
                      uint32_t nrows, uint32_t ncols) {
    clb_dcsr v = matrix_in.view(), out{};
    details::check(clb_dcsr_submatrix(c.get(), &v, i, j, nrows, ncols, &out));
    matrix_out = matrix_dcsr::adopt(c, out);
}

inline void reduce(Controls &c, matrix_dcsr &matrix_out, const matrix_dcsr &matrix_in) {
    clb_dcsr v = matrix_in.view(), out{};
    details::check(clb_dcsr_reduce(c.get(), &v, &out));
    matrix_out = matrix_dcsr::adopt(c, out);
}

// ---- additions without a counterpart in the reference ------------------
// Row-size predictor of the learned single-pass SpGEMM (owns device weights).
class RowSizer {
public:
    explicit RowSizer(Controls &c, uint64_t seed = 1) {
        clb_sizer *s = nullptr;
        details::check(clb_sizer_create(c.get(), seed, &s));
        handle_.reset(s, [](clb_sizer *p) { clb_sizer_destroy(p); });
    }
    RowSizer(Controls &c, const std::vector<float> &params) : RowSizer(c) { set_params(params); }
    std::vector<float> params() const {
        std::vector<float> p((size_t)clb_sizer_num_params());
        details::check(clb_sizer_get_params(handle_.get(), p.data(), p.size()));
        return p;
    }
    void set_params(const std::vector<float> &p) {
        details::check(clb_sizer_set_params(handle_.get(), p.data(), p.size()));
    }
    clb_sizer *get() const { return handle_.get(); }

private:
    std::shared_ptr<clb_sizer> handle_;
};

// C = A*B in one numeric pass sized by the predictor; exact for any predictor.
inline void matrix_multiplication_learned(Controls &c, matrix_dcsr &matrix_out, const matrix_dcsr &a,
                                          const matrix_dcsr &b, const RowSizer &sizer, float margin_log2 = 0.25f,
                                          float slack = 8.0f, clb_spgemm_stats *stats = nullptr,
                                          const clb_spgemm_tuning *tuning = nullptr) {
    clb_dcsr va = a.view(), vb = b.view(), out{};
    details::check(
        clb_dcsr_spgemm_learned(c.get(), &va, &vb, sizer.get(), margin_log2, slack, tuning, &out, stats));
    matrix_out = matrix_dcsr::adopt(c, out);
}

// C = A*B under an accumulator tuning (form 0: exact two-pass, 1: single
// pass into upper-bound slots, 2: exact two-pass keeping the symbolic pass's
// bitmaps for the numeric pass); every tuning gives the same C.
inline void matrix_multiplication_tuned(Controls &c, matrix_dcsr &matrix_out, const matrix_dcsr &a,
                                        const matrix_dcsr &b, const clb_spgemm_tuning &tuning,
                                        clb_spgemm_stats *stats = nullptr) {
    clb_dcsr va = a.view(), vb = b.view(), out{};
    details::check(clb_dcsr_spgemm_tuned(c.get(), &va, &vb, &tuning, &out, stats));
    matrix_out = matrix_dcsr::adopt(c, out);
}

// out[k] = pairs[k].first * pairs[k].second, all pairs in one pass.
inline std::vector<matrix_dcsr> matrix_multiplication_batched(
    Controls &c, const std::vector<std::pair<matrix_dcsr, matrix_dcsr>> &pairs,
    const clb_spgemm_tuning *tuning = nullptr, clb_spgemm_stats *stats = nullptr) {
    std::vector<clb_dcsr> va, vb, vc(pairs.size());
    for (const auto &p : pairs) {
        va.push_back(p.first.view());
        vb.push_back(p.second.view());
    }
    details::check(clb_dcsr_spgemm_batched(c.get(), (uint32_t)pairs.size(), va.data(), vb.data(), vc.data(), tuning,
                                           stats));
    std::vector<matrix_dcsr> out;
    for (auto &m : vc) out.push_back(matrix_dcsr::adopt(c, m));
    return out;
}

// C = A*B written into host memory, in row blocks of A whose copies overlap
// the next block's product (learned form with a sizer, exact form without).
// rows_capacity / cols_capacity bound C's stored rows / entries.
inline matrix_dcsr_cpu matrix_multiplication_to_host(Controls &c, const matrix_dcsr &a, const matrix_dcsr &b,
                                                     uint64_t rows_capacity, uint64_t cols_capacity,
                                                     const RowSizer *sizer = nullptr, uint32_t blocks = 8,
                                                     clb_spgemm_stats *stats = nullptr) {
    clb_dcsr va = a.view(), vb = b.view();
    matrix_dcsr_cpu out;
    out.rpt.resize(rows_capacity + 1);
    out.rows.resize(rows_capacity);
    out.cols.resize(cols_capacity);
    uint64_t nzr = 0, nnz = 0;
    details::check(clb_dcsr_spgemm_to_host(c.get(), &va, &vb, sizer ? sizer->get() : nullptr, 0.25f, 8.0f, nullptr,
                                           blocks, out.rpt.data(), out.rows.data(), out.cols.data(), rows_capacity,
                                           cols_capacity, &nzr, &nnz, stats));
    out.rpt.resize(nzr + 1);
    out.rows.resize(nzr);
    out.cols.resize(nnz);
    return out;
}

// A CUDA graph recorded from the controls' stream: Graph g(c, [&] { ... });
// then g.launch() replays the recorded work.
class Graph {
public:
    template <class F>
    Graph(Controls &c, F &&record) : c_(c) {
        details::check(clb_graph_begin(c.get()));
        void *g = nullptr;
        try {
            record();
        } catch (...) {
            clb_graph_end(c.get(), &g);
            clb_graph_destroy(g);
            throw;
        }
        details::check(clb_graph_end(c.get(), &g));
        g_.reset(g, [](void *p) { clb_graph_destroy(p); });
    }
    void launch() { details::check(clb_graph_launch(c_.get(), g_.get())); }

private:
    Controls c_;
    std::shared_ptr<void> g_;
};

// The host-sync-free batched product (clb_dcsr_spgemm_batched_capture) with
// its buffers sized once from clb_spgemm_batched_plan: enqueue() may be
// recorded into a Graph; result() synchronises and returns each pair's C.
class CapturedBatch {
public:
    CapturedBatch(Controls &c, const std::vector<std::pair<matrix_dcsr, matrix_dcsr>> &pairs,
                  const clb_spgemm_tuning *tuning = nullptr)
        : c_(c), pairs_(pairs) {
        for (const auto &p : pairs) {
            va_.push_back(p.first.view());
            vb_.push_back(p.second.view());
        }
        if (tuning) {
            tuning_ = *tuning;
            has_tuning_ = true;
        }
        details::check(clb_spgemm_batched_plan(c.get(), (uint32_t)pairs.size(), va_.data(), vb_.data(), &rows_, &slots_));
        rpt_ = alloc(c, (rows_ + 1) * 8);
        rws_ = alloc(c, std::max<uint64_t>(rows_, 1) * 4);
        cls_ = alloc(c, std::max<uint64_t>(slots_, 1) * 4);
        res_ = alloc(c, (2 + 2 * (pairs.size() + 1)) * 8);
        flags_ = alloc(c, 4);
    }
    void enqueue() {
        details::check(clb_dcsr_spgemm_batched_capture(
            c_.get(), (uint32_t)pairs_.size(), va_.data(), vb_.data(), has_tuning_ ? &tuning_ : nullptr, slots_,
            (uint64_t *)rpt_.get(), (uint32_t *)rws_.get(), (uint32_t *)cls_.get(), slots_, (uint64_t *)res_.get(),
            (uint32_t *)flags_.get()));
    }
    std::vector<matrix_dcsr_cpu> result() {
        details::check(clb_controls_sync(c_.get()));
        uint32_t flags = 0;
        details::check(clb_memcpy_d2h(c_.get(), &flags, flags_.get(), 4));
        if (flags) throw Exception("captured batch incomplete (capacity exceeded)", CLBOOL_RUN_KERNEL_FAILURE);
        const size_t k = pairs_.size();
        std::vector<uint64_t> r(2 + 2 * (k + 1));
        details::check(clb_memcpy_d2h(c_.get(), r.data(), res_.get(), r.size() * 8));
        std::vector<uint64_t> rpt(r[0] + 1);
        std::vector<uint32_t> rows(r[0]), cols(r[1]);
        details::check(clb_memcpy_d2h(c_.get(), rpt.data(), rpt_.get(), rpt.size() * 8));
        if (r[0]) details::check(clb_memcpy_d2h(c_.get(), rows.data(), rws_.get(), rows.size() * 4));
        if (r[1]) details::check(clb_memcpy_d2h(c_.get(), cols.data(), cls_.get(), cols.size() * 4));
        std::vector<matrix_dcsr_cpu> out(k);
        for (size_t i = 0; i < k; ++i) {
            const uint64_t r0 = r[2 + i], r1 = r[3 + i], j0 = r[3 + k + i], j1 = r[4 + k + i];
            for (uint64_t q = r0; q <= r1; ++q) out[i].rpt.push_back(rpt[q] - j0);
            out[i].rows.assign(rows.begin() + r0, rows.begin() + r1);
            out[i].cols.assign(cols.begin() + j0, cols.begin() + j1);
        }
        return out;
    }

private:
    static Buffer alloc(Controls &c, size_t bytes) {
        void *p = nullptr;
        details::check(clb_malloc(c.get(), bytes, &p));
        return Buffer(c, p, bytes);
    }
    Controls c_;
    std::vector<std::pair<matrix_dcsr, matrix_dcsr>> pairs_;  // keeps the operands alive
    std::vector<clb_dcsr> va_, vb_;
    clb_spgemm_tuning tuning_{};
    bool has_tuning_ = false;
    uint64_t rows_ = 0, slots_ = 0;
    Buffer rpt_, rws_, cls_, res_, flags_;
};
}  // namespace dcsr

namespace coo {
inline void matrix_addition(Controls &c, matrix_coo &matrix_out, const matrix_coo &a, const matrix_coo &b) {
    clb_coo va = a.view(), vb = b.view(), out{};
    details::check(clb_coo_add(c.get(), &va, &vb, &out));
    matrix_out = matrix_coo::adopt(c, out);
}

inline void sort_arrays(Controls &c, Buffer &rows_gpu, Buffer &cols_gpu, uint64_t n) {
    details::check(clb_coo_sort(c.get(), (uint32_t *)rows_gpu.get(), (uint32_t *)cols_gpu.get(), n));
}
}  // namespace coo

namespace csr {
inline void matrix_addition(Controls &c, matrix_csr &out, const matrix_csr &a, const matrix_csr &b) {
    clb_csr va = a.view(), vb = b.view(), o{};
    details::check(clb_csr_add(c.get(), &va, &vb, &o));
    out = matrix_csr::adopt(c, o);
}
}  // namespace csr


// ---- binary DCSR files with a checksum (same format as clbool_b200/io.py) --
// magic "CLBDCSR1" | nrows, ncols, nnz, nzr (u64) | rpt u64[nzr+1] | rows u32[nzr]
// | cols u32[nnz] | SHA-256 of everything before it.  Little-endian hosts.
namespace io {
namespace details {
// SHA-256 (FIPS 180-4).
class Sha256 {
public:
    Sha256() { reset(); }
    void update(const uint8_t *p, size_t n) {
        for (size_t i = 0; i < n; ++i) {
            buf_[len_++ % 64] = p[i];
            if (len_ % 64 == 0) block(buf_);
        }
    }
    void digest(uint8_t out[32]) {
        const uint64_t bits = len_ * 8;
        uint8_t one = 0x80, zero = 0;
        update(&one, 1);
        while (len_ % 64 != 56) update(&zero, 1);
        for (int i = 7; i >= 0; --i) {
            uint8_t b = (uint8_t)(bits >> (8 * i));
            update(&b, 1);
        }
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 4; ++j) out[4 * i + j] = (uint8_t)(h_[i] >> (24 - 8 * j));
    }

private:
    static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
    void reset() {
        static const uint32_t h0[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                       0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
        std::memcpy(h_, h0, sizeof(h_));
        len_ = 0;
    }
    void block(const uint8_t *b) {
        static const uint32_t k[64] = {
            0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
            0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
            0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
            0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
            0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
            0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
            0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
            0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
        uint32_t w[64];
        for (int i = 0; i < 16; ++i)
            w[i] = (uint32_t)b[4 * i] << 24 | (uint32_t)b[4 * i + 1] << 16 | (uint32_t)b[4 * i + 2] << 8 | b[4 * i + 3];
        for (int i = 16; i < 64; ++i) {
            const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
            const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = h_[0], bb = h_[1], c = h_[2], d = h_[3], e = h_[4], f = h_[5], g = h_[6], h = h_[7];
        for (int i = 0; i < 64; ++i) {
            const uint32_t t1 = h + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
            const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & bb) ^ (a & c) ^ (bb & c));
            h = g; g = f; f = e; e = d + t1; d = c; c = bb; bb = a; a = t1 + t2;
        }
        h_[0] += a; h_[1] += bb; h_[2] += c; h_[3] += d; h_[4] += e; h_[5] += f; h_[6] += g; h_[7] += h;
    }
    uint32_t h_[8];
    uint8_t buf_[64];
    uint64_t len_;
};
}  // namespace details

inline void save_dcsr(const std::string &path, uint64_t nrows, uint64_t ncols, const matrix_dcsr_cpu &m) {
    const uint64_t nnz = m.cols.size(), nzr = nnz ? m.rows.size() : 0;
    std::string body("CLBDCSR1");
    auto put = [&](const void *p, size_t n) { body.append((const char *)p, n); };
    const uint64_t hdr[4] = {nrows, ncols, nnz, nzr};
    put(hdr, sizeof(hdr));
    if (nnz) {
        put(m.rpt.data(), 8 * (nzr + 1));
        put(m.rows.data(), 4 * nzr);
        put(m.cols.data(), 4 * nnz);
    }
    uint8_t dg[32];
    details::Sha256 sh;
    sh.update((const uint8_t *)body.data(), body.size());
    sh.digest(dg);
    std::ofstream f(path, std::ios::binary);
    f.write(body.data(), (std::streamsize)body.size());
    f.write((const char *)dg, 32);
    if (!f) throw Exception(path + ": write failed", CLBOOL_INVALID_VALUE);
}

inline matrix_dcsr_cpu load_dcsr(const std::string &path, uint64_t &nrows, uint64_t &ncols) {
    std::ifstream f(path, std::ios::binary);
    std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    if (data.size() < 8 + 32 + 32 || data.compare(0, 8, "CLBDCSR1") != 0)
        throw Exception(path + ": not a DCSR file", CLBOOL_INVALID_VALUE);
    uint8_t dg[32];
    details::Sha256 sh;
    sh.update((const uint8_t *)data.data(), data.size() - 32);
    sh.digest(dg);
    if (std::memcmp(dg, data.data() + data.size() - 32, 32) != 0)
        throw Exception(path + ": checksum mismatch", CLBOOL_INVALID_VALUE);
    uint64_t hdr[4];
    std::memcpy(hdr, data.data() + 8, sizeof(hdr));
    nrows = hdr[0];
    ncols = hdr[1];
    const uint64_t nnz = hdr[2], nzr = hdr[3];
    matrix_dcsr_cpu m;
    if (!nnz) return m;
    if (data.size() != 40 + 8 * (nzr + 1) + 4 * nzr + 4 * nnz + 32)
        throw Exception(path + ": truncated", CLBOOL_INVALID_VALUE);
    const char *p = data.data() + 40;
    m.rpt.resize(nzr + 1);
    m.rows.resize(nzr);
    m.cols.resize(nnz);
    std::memcpy(m.rpt.data(), p, 8 * (nzr + 1));
    std::memcpy(m.rows.data(), p + 8 * (nzr + 1), 4 * nzr);
    std::memcpy(m.cols.data(), p + 8 * (nzr + 1) + 4 * nzr, 4 * nnz);
    return m;
}
}  // namespace io

}  // namespace clbool
