// Host-side output chain of libpned_gpu.so: the reference's TPQ coefficient
// files (Fortran unformatted sequential records) and the canonical
// finite-temperature evaluation of mTPQ runs (eval_mpi).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "pned_internal.h"

using namespace pned;

namespace {

// Largest payload of one subrecord: gfortran's default, 2^31 - 9 bytes
// (its -fmax-subrecord-length); settable for tests.
int64_t g_max_subrecord = 2147483639;

// One Fortran unformatted sequential record (gfortran's documented layout):
// the payload is split into subrecords of at most g_max_subrecord bytes, each
// framed by 4-byte markers holding its length; the leading marker is negated
// when another subrecord follows, the trailing one when a subrecord precedes.
// A record that fits one subrecord is the plain length / payload / length.
bool put_record(FILE *f, const void *data, size_t bytes)
{
    const char *p = static_cast<const char *>(data);
    size_t off = 0;
    do {
        const size_t n = std::min<size_t>(bytes - off, size_t(g_max_subrecord));
        const bool more = off + n < bytes, first = off == 0;
        const int32_t lead = more ? -int32_t(n) : int32_t(n), tail = first ? int32_t(n) : -int32_t(n);
        if (fwrite(&lead, 4, 1, f) != 1 || (n && fwrite(p + off, 1, n, f) != n) || fwrite(&tail, 4, 1, f) != 1)
            return false;
        off += n;
    } while (off < bytes);
    return true;
}

// Reads one record, subrecord by subrecord, into `dst` (capacity `cap` bytes;
// nullptr: only measure); *len receives the record's payload length.  False
// on a malformed record or one longer than cap.
bool read_record(FILE *f, char *dst, size_t cap, size_t *len)
{
    size_t total = 0;
    for (bool first = true;; first = false) {
        int32_t lead = 0, tail = 0;
        if (fread(&lead, 4, 1, f) != 1 || lead == INT32_MIN) return false;
        const size_t n = size_t(lead < 0 ? -int64_t(lead) : int64_t(lead));
        if (dst) {
            if (total + n > cap || (n && fread(dst + total, 1, n, f) != n)) return false;
        } else if (n && std::fseek(f, long(n), SEEK_CUR) != 0) {
            return false;
        }
        total += n;
        if (fread(&tail, 4, 1, f) != 1) return false;
        if (tail != (first ? int32_t(n) : -int32_t(n))) return false;
        if (lead > 0) break;
    }
    *len = total;
    return true;
}

// Reads one record into `out` (resized to the record length).
bool get_record(FILE *f, std::vector<char> &out)
{
    const long pos = std::ftell(f);
    size_t len = 0;
    if (pos < 0 || !read_record(f, nullptr, 0, &len) || std::fseek(f, pos, SEEK_SET) != 0) return false;
    out.resize(len);
    return read_record(f, out.data(), len, &len);
}

// Reads one record of exactly `bytes` bytes into dst.
bool get_record_exact(FILE *f, void *dst, size_t bytes)
{
    size_t len = 0;
    return read_record(f, static_cast<char *>(dst), bytes, &len) && len == bytes;
}

// calc_fac (S_one_half/Hybrid_TPS_eval_mpi.f90:236-281): log-weights of the
// mTPQ states at inverse temperature bt, shifted by their maximum; b is the
// 1-based beta(1..nd1) of one seed.
void calc_fac(int nd1, const double *b, double bt, std::vector<double> &fac1, std::vector<double> &fac2)
{
    fac1.assign(size_t(nd1) + 1, 0.0);
    fac2.assign(size_t(nd1) + 1, 0.0);
    double y = 0.0, maxfac = -1e200;
    for (int i = 1; i <= 2 * (nd1 - 1); ++i) {
        const int m = ((i + 1) >> 1) + 1;
        const double z = std::log(bt / double(2 * i) * b[m - 1]);
        y += z;
        fac1[m] = y;
        maxfac = std::max(y, maxfac);
    }
    for (int i = 1; i <= nd1 - 1; ++i) {
        fac1[i] = std::exp(fac1[i] - maxfac);
        fac2[i] = fac1[i] * bt * b[i] / double(2 * i - 1);
    }
    fac1[nd1] = std::exp(fac1[nd1] - maxfac);
    fac2[nd1] = 0.0;
}

// Sum of v in descending order (lsort, :315-347, then the ordered sums of eval_q).
double sorted_sum(std::vector<double> v)
{
    std::sort(v.begin(), v.end(), std::greater<double>());
    double s = 0.0;
    for (double x : v) s += x;
    return s;
}

// eval_q (:284-313): canonical expectation of dat1 (diagonal) and dat2
// (<k-1|H|k>) terms at bt for one seed.
double eval_q(int nd1, const double *b, const double *dat1, const double *dat2, double bt)
{
    std::vector<double> fac1, fac2;
    calc_fac(nd1, b, bt, fac1, fac2);
    std::vector<double> t1(size_t(nd1) - 1), t2(size_t(nd1) - 1);
    double z = 0.0;
    for (int i = 1; i <= nd1 - 1; ++i) {
        t1[i - 1] = fac1[i] * dat1[i - 1];
        t2[i - 1] = fac2[i] * dat2[i - 1];
        z = z + fac1[i] + fac2[i];
    }
    return (sorted_sum(t1) + sorted_sum(t2)) / z;
}

}  // namespace

extern "C" int pned_write_salphasbeta(const char *path, int num_data1, int num_data2, const double *alpha,
                                      const double *beta, const double *coef)
{
    if (!path || num_data1 < 1 || num_data2 < 1 || !alpha || !beta || !coef)
        return fail(PNED_EINVAL, "pned_write_salphasbeta: bad arguments");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_write_salphasbeta: cannot open ") + path);
    const int32_t n1 = num_data1, n2 = num_data2;
    bool ok = put_record(f, &n1, 4) && put_record(f, &n2, 4) &&
              put_record(f, alpha, sizeof(double) * size_t(n1)) && put_record(f, beta, sizeof(double) * size_t(n1)) &&
              put_record(f, coef, sizeof(double) * size_t(n1) * size_t(n2));
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_write_salphasbeta: write failed");
}

extern "C" int pned_read_salphasbeta(const char *path, int *num_data1, int *num_data2, double *alpha, double *beta,
                                     double *coef, int capacity1)
{
    if (!path || !num_data1 || !num_data2) return fail(PNED_EINVAL, "pned_read_salphasbeta: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_read_salphasbeta: cannot open ") + path);
    std::vector<char> r1, r2, ra, rb, rc;
    bool ok = get_record(f, r1) && r1.size() == 4 && get_record(f, r2) && r2.size() == 4;
    int32_t n1 = 0, n2 = 0;
    if (ok) {
        std::memcpy(&n1, r1.data(), 4);
        std::memcpy(&n2, r2.data(), 4);
        ok = n1 > 0 && n2 > 0;
    }
    if (ok && alpha && beta && coef) {
        ok = capacity1 >= n1 && get_record(f, ra) && ra.size() == sizeof(double) * size_t(n1) && get_record(f, rb) &&
             rb.size() == ra.size() && get_record(f, rc) && rc.size() == sizeof(double) * size_t(n1) * size_t(n2);
        if (ok) {
            std::memcpy(alpha, ra.data(), ra.size());
            std::memcpy(beta, rb.data(), rb.size());
            std::memcpy(coef, rc.data(), rc.size());
        }
    }
    std::fclose(f);
    if (!ok) return fail(PNED_EINVAL, "pned_read_salphasbeta: not a TPQ coefficient file of the expected layout");
    *num_data1 = n1;
    *num_data2 = n2;
    return PNED_OK;
}

extern "C" int pned_tpq_thermo(int num_data1, int n_seeds, const double *beta, const double *energy,
                               const double *hmix, double t_min, double t_max, int num_div, double *out)
{
    if (num_data1 < 2 || n_seeds < 1 || !beta || !energy || !hmix || !out || num_div < 1 || !(t_min > 0) ||
        !(t_max >= t_min))
        return fail(PNED_EINVAL, "pned_tpq_thermo: bad arguments");
    const double lmax = std::log(t_max), lmin = std::log(t_min);
    const double delta = (lmax - lmin) / double(num_div);
    double t_delta = 1e-4;
    if (t_min < t_delta) t_delta = t_min * 0.9;
    std::vector<double> tmp(static_cast<size_t>(n_seeds));
    for (int i1 = 0; i1 <= num_div; ++i1) {
        const double t0 = std::exp(lmin + double(i1) * delta);
        double dat[9];
        for (int i2 = 0; i2 < 3; ++i2) {
            const double bt = i2 == 0 ? 1.0 / (t0 - t_delta) : (i2 == 1 ? 1.0 / t0 : 1.0 / (t0 + t_delta));
            for (int s = 0; s < n_seeds; ++s) {
                const size_t o = size_t(s) * num_data1;
                tmp[s] = eval_q(num_data1, beta + o, energy + o, hmix + o, bt);
            }
            // calc_ave (:349-363)
            double ave = 0.0, var = 0.0;
            for (int s = 0; s < n_seeds; ++s) {
                ave += tmp[s];
                var += tmp[s] * tmp[s];
            }
            ave /= double(n_seeds);
            var = var / double(n_seeds) - ave * ave;
            dat[3 * i2] = bt;
            dat[3 * i2 + 1] = ave;
            dat[3 * i2 + 2] = var;
        }
        // :420-430 (Fortran dat(0:8))
        const double d_e = 0.5 * (dat[7] - dat[1]);
        const double spec = d_e / t_delta;
        const double var_spec = 0.5 * (dat[2] + dat[8]);
        const double spec_d1 = (dat[4] - dat[1]) / t_delta;
        const double spec_d2 = (dat[7] - dat[4]) / t_delta;
        const double del_c = (spec_d2 - spec_d1) / t_delta;
        double *o = out + size_t(i1) * 5;
        o[0] = 1.0 / dat[3];
        o[1] = dat[4];
        o[2] = spec;
        o[3] = var_spec;
        o[4] = del_c;
    }
    return PNED_OK;
}

// ---------------------------------------------------------------------------
// the reference's other output files
// ---------------------------------------------------------------------------
extern "C" int pned_set_max_subrecord(int64_t bytes)
{
    if (bytes < 1 || bytes > 2147483639) return fail(PNED_EINVAL, "pned_set_max_subrecord: 1 .. 2147483639 bytes");
    g_max_subrecord = bytes;
    return PNED_OK;
}

extern "C" int pned_write_vec_data(const char *path, double e, const pned_c128 *x, int64_t ll)
{
    if (!path || !x || ll < 1) return fail(PNED_EINVAL, "pned_write_vec_data: bad arguments");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_write_vec_data: cannot open ") + path);
    bool ok = put_record(f, &e, 8) && put_record(f, x, size_t(ll) * 16);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_write_vec_data: write failed");
}

extern "C" int pned_read_vec_data(const char *path, double *e, pned_c128 *x, int64_t ll)
{
    if (!path || !e || !x || ll < 1) return fail(PNED_EINVAL, "pned_read_vec_data: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_read_vec_data: cannot open ") + path);
    const bool ok = get_record_exact(f, e, 8) && get_record_exact(f, x, size_t(ll) * 16);
    std::fclose(f);
    if (!ok) return fail(PNED_EINVAL, "pned_read_vec_data: not a vector file of this length");
    return PNED_OK;
}

extern "C" int pned_write_dsf_alpha_beta(const char *path, pned_c128 sq, const double *salpha, const double *sbeta,
                                         int s_maxitr)
{
    if (!path || !salpha || !sbeta || s_maxitr < 1) return fail(PNED_EINVAL, "pned_write_dsf_alpha_beta: bad arguments");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_write_dsf_alpha_beta: cannot open ") + path);
    bool ok = put_record(f, &sq, 16) && put_record(f, salpha, sizeof(double) * size_t(s_maxitr)) &&
              put_record(f, sbeta, sizeof(double) * size_t(s_maxitr));
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_write_dsf_alpha_beta: write failed");
}

extern "C" int pned_read_dsf_alpha_beta(const char *path, pned_c128 *sq, double *salpha, double *sbeta, int s_maxitr)
{
    if (!path || !sq || !salpha || !sbeta || s_maxitr < 1)
        return fail(PNED_EINVAL, "pned_read_dsf_alpha_beta: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_read_dsf_alpha_beta: cannot open ") + path);
    std::vector<char> r1, r2, r3;
    const size_t n = sizeof(double) * size_t(s_maxitr);
    const bool ok = get_record(f, r1) && r1.size() == 16 && get_record(f, r2) && r2.size() == n && get_record(f, r3) &&
                    r3.size() == n;
    std::fclose(f);
    if (!ok) return fail(PNED_EINVAL, "pned_read_dsf_alpha_beta: not a DSF coefficient file of this length");
    std::memcpy(sq, r1.data(), 16);
    std::memcpy(salpha, r2.data(), n);
    std::memcpy(sbeta, r3.data(), n);
    return PNED_OK;
}

extern "C" int pned_append_dsf_res(const char *path, double sq_re, const double *q2, const double *w, const double *dsf,
                                   const int *conv, int ll)
{
    if (!path || !q2 || !w || !dsf || !conv || ll < 1) return fail(PNED_EINVAL, "pned_append_dsf_res: bad arguments");
    FILE *f = std::fopen(path, "a");
    if (!f) return fail(PNED_EINVAL, std::string("pned_append_dsf_res: cannot open ") + path);
    // write_dsf_res (S1/2 output.f90:246-264): '(A,F25.18)', then '(2F18.10,2F25.16,I5)' per
    // point, then four list-directed empty records (a single blank each)
    bool ok = std::fprintf(f, "#        %25.18f\n", sq_re) > 0;
    for (int k = 0; k < ll && ok; ++k)
        ok = std::fprintf(f, "%18.10f%18.10f%25.16f%25.16f%5d\n", q2[0], q2[1], w[k], dsf[k], conv[k]) > 0;
    for (int k = 0; k < 4 && ok; ++k) ok = std::fputs(" \n", f) >= 0;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_append_dsf_res: write failed");
}

extern "C" int pned_append_sq(const char *path, int iq, double q1, double q2, double norm_re)
{
    if (!path) return fail(PNED_EINVAL, "pned_append_sq: null path");
    FILE *f = std::fopen(path, "a");
    if (!f) return fail(PNED_EINVAL, std::string("pned_append_sq: cannot open ") + path);
    // the DSF driver's sq.txt line (S1/2 DSF.f90:490-492): '(A,I3,2F12.6,F25.18)'
    bool ok = std::fprintf(f, " q = %3d%12.6f%12.6f%25.18f\n", iq, q1, q2, norm_re) > 0;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_append_sq: write failed");
}

extern "C" int pned_write_dsf_vectors(const char *path, int indx, const pned_c128 *v1, const pned_c128 *v2, int64_t ll)
{
    if (!path || !v1 || !v2 || ll < 1) return fail(PNED_EINVAL, "pned_write_dsf_vectors: bad arguments");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_write_dsf_vectors: cannot open ") + path);
    const int32_t i4 = indx;
    bool ok = put_record(f, &i4, 4) && put_record(f, v1, size_t(ll) * 16) && put_record(f, v2, size_t(ll) * 16);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_write_dsf_vectors: write failed");
}

extern "C" int pned_read_dsf_vectors(const char *path, int *indx, pned_c128 *v1, pned_c128 *v2, int64_t ll)
{
    if (!path || !indx || !v1 || !v2 || ll < 1) return fail(PNED_EINVAL, "pned_read_dsf_vectors: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_read_dsf_vectors: cannot open ") + path);
    const size_t n = size_t(ll) * 16;
    int32_t i4 = 0;
    const bool ok = get_record_exact(f, &i4, 4) && get_record_exact(f, v1, n) && get_record_exact(f, v2, n);
    std::fclose(f);
    if (!ok) return fail(PNED_EINVAL, "pned_read_dsf_vectors: not a DSF vector file of this length");
    *indx = i4;
    return PNED_OK;
}

// ---------------------------------------------------------------------------
// interval_dump / interval_dump_read / check_interval_dump (S1/2 output.f90:50-211)
// ---------------------------------------------------------------------------
extern "C" int pned_write_interval_dump(const char *path, const pned_dump_info *info, const pned_dump_data *d)
{
    if (!path || !info || !d || !d->vec[1] || !d->vec[2] || d->data_size < 1 || d->vec_size < 0)
        return fail(PNED_EINVAL, "pned_write_interval_dump: bad arguments");
    const std::string ipath = std::string(path) + ".info";
    FILE *f = std::fopen(ipath.c_str(), "wb");
    if (!f) return fail(PNED_EINVAL, "pned_write_interval_dump: cannot open " + ipath);
    bool ok = put_record(f, info->dump_name, 128) && put_record(f, &info->np, 4) &&
              put_record(f, info->position, 28) && put_record(f, &info->max_itr, 4) &&
              put_record(f, info->dsf_comp, 2) && put_record(f, &info->s_maxitr, 4) && put_record(f, &info->n, 4) &&
              put_record(f, &info->ibond, 4) && put_record(f, &info->nvec, 4) && put_record(f, &info->total_sz, 4);
    for (int i = 0; i < 12 && ok; ++i) ok = put_record(f, &info->itr_counter[i], 4);
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return fail(PNED_EINVAL, "pned_write_interval_dump: write failed");
    f = std::fopen(path, "wb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_write_interval_dump: cannot open ") + path);
    ok = put_record(f, &d->data_size, 4) && put_record(f, &d->vec_size, 4);
    const double *arr[4] = {d->sa, d->sb, d->sc, d->se};
    const int64_t len[4] = {d->n_sa, d->n_sb, d->n_sc, d->n_se};
    for (int i = 0; i < 4 && ok; ++i)
        if (arr[i]) ok = len[i] >= 0 && put_record(f, arr[i], size_t(len[i]) * 8);
    const size_t vb = size_t(d->data_size) * 16;
    for (int i = 0; i < 5 && ok; ++i)
        if (d->vec[i]) ok = put_record(f, d->vec[i], vb);
    ok = (std::fclose(f) == 0) && ok;
    return ok ? PNED_OK : fail(PNED_EINVAL, "pned_write_interval_dump: write failed");
}

extern "C" int pned_read_interval_dump_info(const char *path, pned_dump_info *info)
{
    if (!path || !info) return fail(PNED_EINVAL, "pned_read_interval_dump_info: bad arguments");
    const std::string ipath = std::string(path) + ".info";
    FILE *f = std::fopen(ipath.c_str(), "rb");
    if (!f) return fail(PNED_EINVAL, "pned_read_interval_dump_info: cannot open " + ipath);
    pned_dump_info t{};
    bool ok = get_record_exact(f, t.dump_name, 128) && get_record_exact(f, &t.np, 4) &&
              get_record_exact(f, t.position, 28) && get_record_exact(f, &t.max_itr, 4) &&
              get_record_exact(f, t.dsf_comp, 2) && get_record_exact(f, &t.s_maxitr, 4) &&
              get_record_exact(f, &t.n, 4) && get_record_exact(f, &t.ibond, 4) && get_record_exact(f, &t.nvec, 4) &&
              get_record_exact(f, &t.total_sz, 4);
    for (int i = 0; i < 12 && ok; ++i) ok = get_record_exact(f, &t.itr_counter[i], 4);
    std::fclose(f);
    if (!ok) return fail(PNED_EINVAL, "pned_read_interval_dump_info: not an interval_dump .info file");
    *info = t;
    return PNED_OK;
}

extern "C" int pned_interval_dump_records(const char *path, int64_t *bytes, int cap, int *count)
{
    if (!path || !count || cap < 0 || (cap && !bytes)) return fail(PNED_EINVAL, "pned_interval_dump_records: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_interval_dump_records: cannot open ") + path);
    int n = 0;
    bool ok = true;
    for (;;) {
        const int c = std::fgetc(f);
        if (c == EOF) break;
        std::ungetc(c, f);
        size_t len = 0;
        if (!read_record(f, nullptr, 0, &len)) { ok = false; break; }
        if (n < cap) bytes[n] = int64_t(len);
        ++n;
    }
    std::fclose(f);
    if (!ok) return fail(PNED_EINVAL, "pned_interval_dump_records: malformed record");
    *count = n;
    return PNED_OK;
}

extern "C" int pned_read_interval_dump(const char *path, pned_dump_data *d)
{
    if (!path || !d || !d->vec[1] || !d->vec[2]) return fail(PNED_EINVAL, "pned_read_interval_dump: bad arguments");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(PNED_EINVAL, std::string("pned_read_interval_dump: cannot open ") + path);
    int32_t ds = 0, vs = 0;
    bool ok = get_record_exact(f, &ds, 4) && get_record_exact(f, &vs, 4) && ds >= 1 &&
              (d->data_size <= 0 || ds == d->data_size);
    double *arr[4] = {d->sa, d->sb, d->sc, d->se};
    const int64_t len[4] = {d->n_sa, d->n_sb, d->n_sc, d->n_se};
    for (int i = 0; i < 4 && ok; ++i)
        if (arr[i]) ok = len[i] >= 0 && get_record_exact(f, arr[i], size_t(len[i]) * 8);
    for (int i = 0; i < 5 && ok; ++i)
        if (d->vec[i]) ok = get_record_exact(f, d->vec[i], size_t(ds) * 16);
    std::fclose(f);
    if (!ok) return fail(PNED_EINVAL, "pned_read_interval_dump: records do not match the expected arrays");
    d->data_size = ds;
    d->vec_size = vs;
    return PNED_OK;
}
