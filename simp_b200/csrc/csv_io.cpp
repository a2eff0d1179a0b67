// The reference's snapshot files, written from a context's device state and
// read back for a spin-up:
//   particle_momentum.csv  i, x/1000, y/1000, 100 vx, 100 vy      (format 1001)
//   particle_state.csv     i, mass, p, hsml, A, h, eps11, eps12, eps22,
//                          sig11, sig12, sig22                      (format 1002)
//   particle_other.csv     ntotal, ntotalb, current_time / 3600    (format 1003)
// (in_out/output.f90:61-78; created empty by initialize.f90:83-95), and
//   boundary_particles.csv j, xb/1000, yb/1000, massb  (boundaries.f90:31, 52-63).
// Every output call appends one snapshot.  The reference's spin-up reader
// (initialize.f90:234-330) reads 14 columns per state record where the
// writer writes 11, and always the first snapshot; simp_csv_read_snapshot
// reads the 11 written columns of any snapshot.
//
// Host code: output is rare (every save_step), and the text is formatted on
// the host cores in parallel from one device-to-host copy of the state.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "simp_gpu.h"

namespace {

thread_local std::string g_err;

int csv_fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

// Right-justifies s in a field of width w, or fills it with '*' when it does
// not fit (Fortran output editing).
void put_field(std::string &out, const char *s, int len, int w) {
    if (len > w) {
        out.append((size_t)w, '*');
        return;
    }
    out.append((size_t)(w - len), ' ');
    out.append(s, (size_t)len);
}

// Iw.
void put_int(std::string &out, long long v, int w) {
    char b[32];
    const int n = std::snprintf(b, sizeof b, "%lld", v);
    put_field(out, b, n, w);
}

// Ew.d and Ew.dEe as gfortran writes them: a mantissa 0.d1..dd (rounded to
// nearest), the exponent as E+xx (e = 0: two digits, or +xxx without the E
// above 99) or E+x..x with e digits, and the optional leading zero only
// when the field has room for it.
void put_E(std::string &out, double v, int w, int d, int e) {
    char core[64];
    int len = 0;
    const bool neg = std::signbit(v);
    if (std::isnan(v)) {
        put_field(out, "NaN", 3, w);
        return;
    }
    if (std::isinf(v)) {
        const char *s = neg ? "-Infinity" : "Infinity";
        put_field(out, s, (int)std::strlen(s), w);
        return;
    }
    char digits[40];
    int x10 = 0;
    if (v == 0.0) {
        std::memset(digits, '0', (size_t)d);
    } else {
        // d significant digits: D.DDDDe+X gives 0.DDDDD x 10^(X+1)
        char b[64];
        std::snprintf(b, sizeof b, "%.*e", d - 1, std::fabs(v));
        int k = 0;
        for (const char *p = b; *p && *p != 'e'; ++p)
            if (*p != '.') digits[k++] = *p;
        x10 = std::atoi(std::strchr(b, 'e') + 1) + 1;
    }
    core[len++] = '.';
    std::memcpy(core + len, digits, (size_t)d);
    len += d;
    const int ax = std::abs(x10);
    if (e > 0) {
        char eb[16];
        const int n = std::snprintf(eb, sizeof eb, "%0*d", e, ax);
        if (n > e) {
            out.append((size_t)w, '*');
            return;
        }
        core[len++] = 'E';
        core[len++] = x10 < 0 ? '-' : '+';
        std::memcpy(core + len, eb, (size_t)n);
        len += n;
    } else if (ax <= 99) {
        len += std::snprintf(core + len, sizeof core - (size_t)len, "E%c%02d", x10 < 0 ? '-' : '+', ax);
    } else {
        len += std::snprintf(core + len, sizeof core - (size_t)len, "%c%03d", x10 < 0 ? '-' : '+', ax);
    }
    char full[80];
    int n = 0;
    if (neg) full[n++] = '-';
    if (len + n + 1 <= w) full[n++] = '0';
    std::memcpy(full + n, core, (size_t)len);
    n += len;
    put_field(out, full, n, w);
}

// " , " followed by E15.8E3: one (1x, A1, 1x, e15.8E3) group.
void put_col(std::string &out, double v) {
    out.append(" , ");
    put_E(out, v, 15, 8, 3);
}

// Formats records [0, n) with f(i, out) on the host's cores and appends them
// to the file, in order.
template <class F>
int append_records(const std::string &path, int n, F &&f) {
    const int nt = std::max(1, std::min((int)std::thread::hardware_concurrency(), std::max(1, n / 4096)));
    std::vector<std::string> parts((size_t)nt);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) {
        th.emplace_back([&, t]() {
            const int i0 = (int)((long long)n * t / nt), i1 = (int)((long long)n * (t + 1) / nt);
            std::string &s = parts[(size_t)t];
            s.reserve((size_t)(i1 - i0) * 200);
            for (int i = i0; i < i1; ++i) f(i, s);
        });
    }
    for (auto &x : th) x.join();
    FILE *fp = std::fopen(path.c_str(), "a");
    if (!fp) return csv_fail(SIMP_ERR_BADARG, "cannot open " + path + " for appending: " + std::strerror(errno));
    bool ok = true;
    for (const std::string &s : parts) ok = ok && std::fwrite(s.data(), 1, s.size(), fp) == s.size();
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return csv_fail(SIMP_ERR_BADARG, "write failed: " + path);
    return SIMP_OK;
}

std::string join(const char *folder, const char *name) {
    std::string p = folder ? folder : "";
    if (!p.empty() && p.back() != '/') p += '/';
    return p + name;
}

// Lines [first, first + count) of a text file (without their newlines;
// count < 0: to the end), streamed: a file of many snapshots is never held
// in memory whole.
int read_lines(const std::string &path, std::vector<std::string> *lines, long long first = 0,
               long long count = -1) {
    FILE *fp = std::fopen(path.c_str(), "r");
    if (!fp) return csv_fail(SIMP_ERR_BADARG, "cannot open " + path + ": " + std::strerror(errno));
    lines->clear();
    std::string cur;
    long long line = 0;
    const long long last = (count < 0) ? -1 : first + count;
    char buf[1 << 16];
    size_t got;
    bool done = false;
    while (!done && (got = std::fread(buf, 1, sizeof buf, fp)) > 0) {
        for (size_t k = 0; k < got; ++k) {
            if (buf[k] == '\n') {
                if (line >= first) lines->push_back(cur);
                cur.clear();
                if (++line == last) {
                    done = true;
                    break;
                }
            } else if (buf[k] != '\r' && line >= first) {
                cur.push_back(buf[k]);
            }
        }
    }
    if (!done && !cur.empty() && line >= first) lines->push_back(cur);
    std::fclose(fp);
    return SIMP_OK;
}

// List-directed read of up to `want` numbers separated by commas or blanks.
int parse_numbers(const std::string &line, double *v, int want) {
    const char *p = line.c_str();
    int k = 0;
    while (k < want) {
        while (*p == ' ' || *p == ',' || *p == '\t') ++p;
        if (!*p) break;
        char *end = nullptr;
        const double x = std::strtod(p, &end);
        if (end == p) break;
        v[k++] = x;
        p = end;
    }
    return k;
}

}  // namespace

extern "C" {

const char *simp_csv_last_error(void) { return g_err.c_str(); }

int32_t simp_csv_create_output(const char *folder) {
    for (const char *name : {"particle_momentum.csv", "particle_state.csv", "particle_other.csv"}) {
        const std::string path = join(folder, name);
        FILE *fp = std::fopen(path.c_str(), "w");
        if (!fp) return csv_fail(SIMP_ERR_BADARG, "cannot create " + path + ": " + std::strerror(errno));
        std::fclose(fp);
    }
    return SIMP_OK;
}

int32_t simp_csv_append_snapshot(const char *folder, int32_t ntotal, int32_t ntotalb, double current_time,
                                 const double *x, const double *vx, const double *mass, const double *p,
                                 const double *hsml, const double *A, const double *h, const double *eps11,
                                 const double *eps12, const double *eps22, const double *sig11,
                                 const double *sig12, const double *sig22) {
    if (ntotal < 0 || (ntotal > 0 && (!x || !vx || !mass || !p || !hsml || !A || !h || !eps11 || !eps12 ||
                                      !eps22 || !sig11 || !sig12 || !sig22)))
        return csv_fail(SIMP_ERR_BADARG, "append_snapshot: bad sizes or null arrays");
    int rc = append_records(join(folder, "particle_momentum.csv"), ntotal, [&](int i, std::string &s) {
        s.push_back(' ');
        put_int(s, i + 1, 7);
        for (int d = 0; d < 2; ++d) put_col(s, x[2 * (size_t)i + d] / 1000);
        for (int d = 0; d < 2; ++d) put_col(s, vx[2 * (size_t)i + d] * 100);
        s.push_back('\n');
    });
    if (rc) return rc;
    rc = append_records(join(folder, "particle_state.csv"), ntotal, [&](int i, std::string &s) {
        s.push_back(' ');
        put_int(s, i + 1, 7);
        for (const double *a : {mass, p, hsml, A, h, eps11, eps12, eps22, sig11, sig12, sig22}) put_col(s, a[i]);
        s.push_back('\n');
    });
    if (rc) return rc;
    return append_records(join(folder, "particle_other.csv"), 1, [&](int, std::string &s) {
        s.push_back(' ');
        put_int(s, ntotal, 7);
        s.append(" , ");
        put_int(s, ntotalb, 7);
        s.append(" , ");
        put_E(s, current_time / 3600, 15, 8, 3);
        s.push_back('\n');
    });
}

int32_t simp_csv_write_walls(const char *folder, int32_t ntotalb, const double *xb, const double *massb) {
    if (ntotalb < 0 || (ntotalb > 0 && (!xb || !massb)))
        return csv_fail(SIMP_ERR_BADARG, "write_walls: bad sizes or null arrays");
    const std::string path = join(folder, "boundary_particles.csv");
    FILE *fp = std::fopen(path.c_str(), "w");
    if (!fp) return csv_fail(SIMP_ERR_BADARG, "cannot create " + path + ": " + std::strerror(errno));
    std::fclose(fp);
    return append_records(path, ntotalb, [&](int j, std::string &s) {
        s.push_back(' ');
        put_int(s, j + 1, 5);
        for (int d = 0; d < 2; ++d) {
            s.append(" , ");
            put_E(s, xb[2 * (size_t)j + d] / 1000, 14, 8, 0);
        }
        s.append(" , ");
        put_E(s, massb[j], 14, 8, 0);
        s.push_back('\n');
    });
}

int32_t simp_csv_read_snapshot(const char *folder, int32_t snapshot, int32_t cap, int32_t *ntotal,
                               int32_t *ntotalb, double *current_time, double *x, double *vx, double *mass,
                               double *p, double *hsml, double *A, double *h) {
    std::vector<std::string> other, mom, st;
    int rc = read_lines(join(folder, "particle_other.csv"), &other);
    if (rc) return rc;
    std::vector<long long> n_of;
    std::vector<double> nb_of, t_of;
    for (const std::string &l : other) {
        double v[3];
        if (parse_numbers(l, v, 3) == 3) {
            n_of.push_back((long long)v[0]);
            nb_of.push_back(v[1]);
            t_of.push_back(v[2]);
        }
    }
    const int ns = (int)n_of.size();
    if (ns == 0) return csv_fail(SIMP_ERR_BADARG, "read_snapshot: no snapshot in particle_other.csv");
    const int k = snapshot < 0 ? ns + snapshot : snapshot;
    if (k < 0 || k >= ns) return csv_fail(SIMP_ERR_BADARG, "read_snapshot: no snapshot " + std::to_string(snapshot));
    long long first = 0;
    for (int q = 0; q < k; ++q) first += n_of[(size_t)q];
    const long long n = n_of[(size_t)k];
    if (ntotal) *ntotal = (int32_t)n;
    if (ntotalb) *ntotalb = (int32_t)nb_of[(size_t)k];
    if (current_time) *current_time = t_of[(size_t)k] * 3600;   // initialize.f90:285
    if (!x && !vx && !mass && !p && !hsml && !A && !h) return SIMP_OK;   // sizes only
    if (n > cap)
        return csv_fail(SIMP_ERR_MAXN, "The number of particles read from the input file is higher than the "
                                       "maximum allowed. (initialize.f90:276-283)");
    if ((rc = read_lines(join(folder, "particle_momentum.csv"), &mom, first, n))) return rc;
    if ((rc = read_lines(join(folder, "particle_state.csv"), &st, first, n))) return rc;
    if ((long long)mom.size() < n || (long long)st.size() < n)
        return csv_fail(SIMP_ERR_BADARG, "read_snapshot: the particle files end before snapshot " +
                                             std::to_string(k));
    for (long long r = first; r < first + n; ++r) {
        double a[5], b[12];
        if (parse_numbers(mom[(size_t)(r - first)], a, 5) != 5 || parse_numbers(st[(size_t)(r - first)], b, 12) != 12)
            return csv_fail(SIMP_ERR_BADARG, "read_snapshot: short record at line " + std::to_string(r + 1));
        const long long i = (long long)a[0] - 1;
        if (i < 0 || i >= n || (long long)b[0] - 1 != i)
            return csv_fail(SIMP_ERR_BADARG, "read_snapshot: bad particle index at line " + std::to_string(r + 1));
        // km -> m and cm/s -> m/s, initialize.f90:304-306
        if (x) { x[2 * i] = a[1] * 1000; x[2 * i + 1] = a[2] * 1000; }
        if (vx) { vx[2 * i] = a[3] / 100; vx[2 * i + 1] = a[4] / 100; }
        if (mass) mass[i] = b[1];
        if (p) p[i] = b[2];
        if (hsml) hsml[i] = b[3];
        if (A) A[i] = b[4];
        if (h) h[i] = b[5];
    }
    return SIMP_OK;
}

int32_t simp_csv_read_walls(const char *folder, int32_t cap, int32_t *ntotalb, double *xb, double *massb) {
    std::vector<std::string> lines;
    int rc = read_lines(join(folder, "boundary_particles.csv"), &lines);
    if (rc) return rc;
    std::vector<std::string> recs;
    for (const std::string &l : lines)
        if (l.find_first_not_of(" \t") != std::string::npos) recs.push_back(l);
    const int nb = (int)recs.size();
    if (ntotalb) *ntotalb = nb;
    if (!xb && !massb) return SIMP_OK;
    if (nb > cap)
        return csv_fail(SIMP_ERR_MAXN, "The number of boundary particles read from the input file is higher "
                                       "than the maximum allowed. (boundaries.f90:136-143)");
    for (int r = 0; r < nb; ++r) {
        double a[4];
        if (parse_numbers(recs[(size_t)r], a, 4) != 4)
            return csv_fail(SIMP_ERR_BADARG, "read_walls: short record at line " + std::to_string(r + 1));
        const long long j = (long long)a[0] - 1;
        if (j < 0 || j >= nb) return csv_fail(SIMP_ERR_BADARG, "read_walls: bad index at line " + std::to_string(r + 1));
        if (xb) { xb[2 * j] = a[1] * 1000; xb[2 * j + 1] = a[2] * 1000; }   // boundaries.f90:152
        if (massb) massb[j] = a[3];
    }
    return SIMP_OK;
}

}  // extern "C"
