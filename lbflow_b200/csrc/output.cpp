// output.cpp -- the reference's CSV text formats, formatted on all host cores.
//
// Output steps of the reference write every node's density, velocity and scalar
// as `{:.8e}` text (src/momentum/io.rs:112-192, src/passive_scalar/io.rs:76-108)
// and, once, the node coordinates (src/momentum/io.rs:194-224).  Text formatting
// dominates those steps, so it is done here in parallel chunks with
// std::to_chars (exact shortest-round-trip machinery, correctly rounded) and then
// rewritten into Rust's exponent style: no '+', no zero padding ("1.00000000e0",
// "-2.50000000e-5"); NaN prints as "NaN" and infinities as "inf" / "-inf", as
// Rust's formatter does.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lbflow.h"

lbf_status lbf_internal_fail(lbf_status s, const char* msg);   // abi.cu

namespace {

constexpr int MAX_FIELD = 24;   // longest "{:.8e}" field: "-1.23456789e-308" (16) with room

// Writes Rust's `{:.8e}` of v at p; returns the number of characters.
int rust_e8(double v, char* p) {
    if (std::isnan(v)) { std::memcpy(p, "NaN", 3); return 3; }
    if (std::isinf(v)) {
        if (v < 0) { std::memcpy(p, "-inf", 4); return 4; }
        std::memcpy(p, "inf", 3); return 3;
    }
    char tmp[40];
    auto r = std::to_chars(tmp, tmp + sizeof(tmp), v, std::chars_format::scientific, 8);
    const int len = (int)(r.ptr - tmp);
    const char* e = (const char*)std::memchr(tmp, 'e', len);
    const int mant = (int)(e - tmp);
    std::memcpy(p, tmp, mant + 1);   // mantissa and 'e'
    int k = mant + 1;
    const char* q = e + 1;
    if (*q == '-') p[k++] = *q++;
    else if (*q == '+') ++q;
    while (*q == '0' && q + 1 < tmp + len) ++q;   // drop leading zeros of the exponent
    while (q < tmp + len) p[k++] = *q++;
    return k;
}

int write_int(long long v, char* p) {
    auto r = std::to_chars(p, p + 24, v);
    return (int)(r.ptr - p);
}

int thread_count(int32_t threads, long long rows) {
    int t = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    return (int)std::max<long long>(1, std::min<long long>(t, (rows + 4095) / 4096));
}

// Formats rows [r0, r1) with fmt_row into one string per chunk, then joins them.
template <class RowFn>
lbf_status format_rows(long long rows, int row_max, int32_t threads, char* out, int64_t cap, int64_t* len,
                       RowFn fmt_row) {
    const int nt = thread_count(threads, rows);
    std::vector<std::string> part(nt);
    auto work = [&](int t) {
        const long long r0 = rows * t / nt, r1 = rows * (t + 1) / nt;
        std::string& s = part[t];
        s.resize((size_t)(r1 - r0) * row_max);
        char* p = s.data();
        for (long long r = r0; r < r1; ++r) p += fmt_row(r, p);
        s.resize((size_t)(p - s.data()));
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    int64_t total = 0;
    for (auto& s : part) total += (int64_t)s.size();
    if (len) *len = total;
    if (!out) return LBF_OK;   // size query
    if (total > cap) return lbf_internal_fail(LBF_EINVAL, "lbf_format: output buffer too small (see *len)");
    char* p = out;
    for (auto& s : part) { std::memcpy(p, s.data(), s.size()); p += s.size(); }
    return LBF_OK;
}

}  // namespace

extern "C" lbf_status lbf_format_csv(const double* values, int64_t rows, int32_t cols, char* out, int64_t cap,
                                     int64_t* len, int32_t threads) {
    if (rows < 0 || cols < 1 || cols > 64 || (rows > 0 && !values))
        return lbf_internal_fail(LBF_EINVAL, "lbf_format_csv: need rows >= 0, 1 <= cols <= 64, values");
    const int row_max = cols * (MAX_FIELD + 1) + 1;
    return format_rows(rows, row_max, threads, out, cap, len, [&](long long r, char* p) {
        const double* v = values + r * cols;
        int k = 0;
        for (int c = 0; c < cols; ++c) {
            if (c) p[k++] = ',';
            k += rust_e8(v[c], p + k);
        }
        p[k++] = '\n';
        return k;
    });
}

extern "C" lbf_status lbf_format_coordinates(const int64_t* n, int32_t d, double delta_x, const uint8_t* node_type,
                                             char* out, int64_t cap, int64_t* len, int32_t threads) {
    if (!n || (d != 2 && d != 3)) return lbf_internal_fail(LBF_EINVAL, "lbf_format_coordinates: d must be 2 or 3");
    const long long nx = n[0], ny = n[1], nz = d == 3 ? n[2] : 1;
    if (nx < 1 || ny < 1 || nz < 1) return lbf_internal_fail(LBF_EINVAL, "lbf_format_coordinates: bad size");
    const long long rows = nx * ny * nz;
    const int row_max = 3 * 21 + 3 * (MAX_FIELD + 1) + 8;
    return format_rows(rows, row_max, threads, out, cap, len, [&](long long r, char* p) {
        const long long idx[3] = {r % nx, (r / nx) % ny, r / (nx * ny)};
        int k = 0;
        for (int a = 0; a < d; ++a) { k += write_int(idx[a], p + k); p[k++] = ','; }
        // node-centred coordinates (src/momentum/lattice.rs:86-89)
        for (int a = 0; a < d; ++a) { k += rust_e8(((double)idx[a] + 0.5) * delta_x, p + k); p[k++] = ','; }
        const bool solid = node_type && node_type[r];
        std::memcpy(p + k, solid ? "solid\n" : "fluid\n", 6);
        return k + 6;
    });
}
