// host_layer_check.cpp -- drives the C++ host layer (include/clbool/clbool.hpp)
// the way the reference's example test does (test/test_operations.cpp:279-319)
// and checks the results: the README matrices, then random products and sums
// against a std::set restatement of the boolean semiring.  Exits non-zero on
// any mismatch; prints "host layer OK" on success.
#include <clbool/clbool.hpp>

#include <algorithm>
#include <cstdio>
#include <random>
#include <set>

using namespace clbool;

static int failures = 0;
#define EXPECT(cond)                                                    \
    do {                                                                \
        if (!(cond)) {                                                  \
            std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond); \
            ++failures;                                                 \
        }                                                               \
    } while (0)

static matrix_coo_cpu_pairs random_pairs(uint32_t n, uint32_t count, uint32_t seed) {
    std::mt19937 rng(seed);
    std::set<coordinates> s;
    for (uint32_t i = 0; i < count; ++i) s.insert({rng() % n, rng() % n});
    return matrix_coo_cpu_pairs(s.begin(), s.end());
}

static matrix_dcsr_cpu dcsr_of(const matrix_coo_cpu_pairs &p) {
    matrix_dcsr_cpu m;
    for (size_t i = 0; i < p.size(); ++i) {
        if (i == 0 || p[i].first != p[i - 1].first) {
            m.rpt.push_back(i);
            m.rows.push_back(p[i].first);
        }
        m.cols.push_back(p[i].second);
    }
    m.rpt.push_back(p.size());
    if (p.empty()) m.rpt.clear();
    return m;
}

static matrix_coo_cpu_pairs product(const matrix_coo_cpu_pairs &a, const matrix_coo_cpu_pairs &b) {
    std::set<coordinates> out;
    for (auto &x : a)
        for (auto it = std::lower_bound(b.begin(), b.end(), coordinates{x.second, 0});
             it != b.end() && it->first == x.second; ++it)
            out.insert({x.first, it->second});
    return matrix_coo_cpu_pairs(out.begin(), out.end());
}

static matrix_coo_cpu_pairs pairs_of(const matrix_dcsr_cpu &m) {
    matrix_coo_cpu_pairs p;
    for (size_t r = 0; r + 1 < m.rpt.size(); ++r)
        for (uint64_t j = m.rpt[r]; j < m.rpt[r + 1]; ++j) p.push_back({m.rows[r], m.cols[j]});
    return p;
}

int main(int argc, char **argv) {
    Controls controls = create_controls();
    show_devices();

    // ---- the reference's example (README.md:55-92) ----
    std::vector<uint32_t> a_rows = {0, 0, 0, 2, 2, 4}, a_cols = {0, 1, 4, 2, 3, 2};
    std::vector<uint32_t> b_rows = {1, 1, 2, 3, 3, 3, 5}, b_cols = {0, 4, 2, 2, 3, 4, 2};
    matrix_coo a_coo(controls, a_rows.data(), a_cols.data(), 5, 5, 6);
    matrix_coo b_coo(controls, b_rows.data(), b_cols.data(), 5, 5, 7);
    matrix_coo c_coo;
    coo::matrix_addition(controls, c_coo, a_coo, b_coo);
    EXPECT(c_coo.nnz() == 12);
    matrix_dcsr a_dcsr = coo_to_dcsr_shallow(controls, a_coo);
    matrix_dcsr b_dcsr = coo_to_dcsr_shallow(controls, b_coo);
    EXPECT(a_dcsr.cols_gpu().get() == a_coo.cols_gpu().get());  // shallow for cols
    matrix_dcsr c_dcsr;
    dcsr::matrix_multiplication_hash(controls, c_dcsr, a_dcsr, b_dcsr);
    matrix_dcsr_cpu h = matrix_dcsr_from_gpu(controls, c_dcsr);
    EXPECT((h.rpt == std::vector<uint64_t>{0, 2, 5, 6}));
    EXPECT((h.rows == cpu_buffer{0, 2, 4}));
    EXPECT((h.cols == cpu_buffer{0, 4, 2, 3, 4, 2}));
    dcsr::kronecker_product(controls, c_dcsr, a_dcsr, b_dcsr);
    EXPECT(c_dcsr.nnz() == 42 && c_dcsr.nrows() == 25);
    matrix_csr a_csr = dcsr_to_csr(controls, a_dcsr);
    matrix_csr b_csr = dcsr_to_csr(controls, a_dcsr);
    matrix_csr c_csr;
    csr::matrix_addition(controls, c_csr, a_csr, b_csr);
    EXPECT(c_csr.nnz() == a_dcsr.nnz());

    // ---- random products and sums ----
    for (uint32_t seed = 1; seed <= 6; ++seed) {
        uint32_t n = 50 + 400 * seed;
        auto pa = random_pairs(n, n * (2 + seed), seed);
        auto pb = random_pairs(n, n * 3, seed + 100);
        matrix_dcsr A = matrix_dcsr_from_cpu(controls, dcsr_of(pa), n);
        matrix_dcsr B = matrix_dcsr_from_cpu(controls, dcsr_of(pb), n);
        matrix_dcsr C;
        dcsr::matrix_multiplication_hash(controls, C, A, B);
        EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, C)) == product(pa, pb));
        matrix_dcsr C2;
        dcsr::matrix_multiplication(controls, C2, A, B);
        EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, C2)) == product(pa, pb));
        // additions without a reference counterpart: learned and batched forms
        dcsr::RowSizer sizer(controls, seed);
        matrix_dcsr C3;
        dcsr::matrix_multiplication_learned(controls, C3, A, B, sizer);
        EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, C3)) == product(pa, pb));
        {  // the two-pass form keeping its symbolic pass's bitmaps
            clb_spgemm_tuning kept;
            clb_spgemm_tuning_default(&kept);
            kept.form = 2;
            kept.bitmap_min = 256;  // bitmap rows even in this small product
            matrix_dcsr C4;
            dcsr::matrix_multiplication_tuned(controls, C4, A, B, kept);
            EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, C4)) == product(pa, pb));
        }
        auto batch = dcsr::matrix_multiplication_batched(controls, {{A, B}, {B, A}, {A, A}});
        EXPECT(batch.size() == 3);
        EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, batch[0])) == product(pa, pb));
        EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, batch[1])) == product(pb, pa));
        EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, batch[2])) == product(pa, pa));
        // C written straight into host memory, in 3 row blocks
        {
            matrix_dcsr_cpu h = dcsr::matrix_multiplication_to_host(controls, A, B, n, (uint64_t)n * n, &sizer, 3);
            matrix_dcsr_cpu w = matrix_dcsr_from_gpu(controls, C);
            EXPECT(h.rpt == w.rpt && h.rows == w.rows && h.cols == w.cols);
        }
        // the host-sync-free batch, recorded into a CUDA graph and replayed twice
        {
            dcsr::CapturedBatch cap(controls, {{A, B}, {B, A}});
            dcsr::Graph graph(controls, [&] { cap.enqueue(); });
            for (int rep = 0; rep < 2; ++rep) {
                graph.launch();
                auto got = cap.result();
                EXPECT(got.size() == 2);
                matrix_dcsr_cpu w0 = matrix_dcsr_from_gpu(controls, batch[0]);
                matrix_dcsr_cpu w1 = matrix_dcsr_from_gpu(controls, batch[1]);
                EXPECT(got[0].rpt == w0.rpt && got[0].rows == w0.rows && got[0].cols == w0.cols);
                EXPECT(got[1].rpt == w1.rpt && got[1].rows == w1.rows && got[1].cols == w1.cols);
            }
        }

        std::vector<uint32_t> ar, ac, br, bc;
        for (auto &p : pa) { ar.push_back(p.first); ac.push_back(p.second); }
        for (auto &p : pb) { br.push_back(p.first); bc.push_back(p.second); }
        matrix_coo CA(controls, ar.data(), ac.data(), n, n, ar.size());
        matrix_coo CB(controls, br.data(), bc.data(), n, n, br.size());
        matrix_coo S;
        coo::matrix_addition(controls, S, CA, CB);
        std::set<coordinates> u(pa.begin(), pa.end());
        u.insert(pb.begin(), pb.end());
        matrix_coo_cpu hs = matrix_coo_from_gpu(controls, S);
        matrix_coo_cpu_pairs got;
        for (size_t i = 0; i < hs.rows.size(); ++i) got.push_back({hs.rows[i], hs.cols[i]});
        EXPECT(got == matrix_coo_cpu_pairs(u.begin(), u.end()));
    }

    // ---- binary DCSR files: written here, read back here and (with argv[1])
    // left for the Python reader to check the shared format ----
    {
        const std::string path = argc > 1 ? argv[1] : "/tmp/clbool_b200_check.dcsr";
        matrix_dcsr_cpu h = matrix_dcsr_from_gpu(controls, a_dcsr);
        io::save_dcsr(path, 5, 5, h);
        uint64_t nr = 0, nc = 0;
        matrix_dcsr_cpu back = io::load_dcsr(path, nr, nc);
        EXPECT(nr == 5 && nc == 5 && back.rpt == h.rpt && back.rows == h.rows && back.cols == h.cols);
        matrix_dcsr dev = matrix_dcsr_from_cpu(controls, back, 5);
        EXPECT(pairs_of(matrix_dcsr_from_gpu(controls, dev)) == pairs_of(h));
    }

    // ---- errors surface as clbool::Exception with the reference's Status ----
    try {
        matrix_dcsr bad(7, 7), out;
        dcsr::matrix_multiplication_hash(controls, out, a_dcsr, bad);
        EXPECT(false);
    } catch (const Exception &e) {
        EXPECT(e.status() == CLBOOL_INVALID_ARGUMENT);
    }
    try {
        create_controls(0, 1000);
        EXPECT(false);
    } catch (const Exception &e) {
        EXPECT(e.status() == CLBOOL_CREATE_CONTROLS_ERROR);
    }

    if (failures) {
        std::fprintf(stderr, "%d check(s) failed\n", failures);
        return 1;
    }
    std::printf("host layer OK\n");
    return 0;
}
