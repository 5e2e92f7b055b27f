// State files (io.f90:98-392): the netCDF-3 files io_save_state writes and
// io_load_state reads, with radial interpolation onto another mesh and
// re-truncation to other K, M.
//
// libnetcdf is not used: the file format (netCDF classic, "CDF1", and the
// 64-bit offset variant, "CDF2"; CDF5 is read too) is a published
// specification, and the few structures a state file holds are written and
// parsed here.  All numbers in the file are big-endian.
//
// A state file has dimensions r (N), H (harmonics) and ReIm (2); global
// attributes t, Re, alpha (double); variables r(r), dt, dtcor, dtcfl
// (scalars) and Ur, Ut, Uz(ReIm, H, r) (C order, r fastest) with integer
// attributes K, M, Mp (io.f90:327-378).
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>
#include "pf_internal.cuh"

namespace {

enum NcType { NC_BYTE = 1, NC_CHAR = 2, NC_SHORT = 3, NC_INT = 4, NC_FLOAT = 5, NC_DOUBLE = 6,
              NC_UBYTE = 7, NC_USHORT = 8, NC_UINT = 9, NC_INT64 = 10, NC_UINT64 = 11 };
constexpr uint32_t TAG_DIM = 0x0A, TAG_VAR = 0x0B, TAG_ATT = 0x0C;

int type_size(int t) {
    switch (t) {
    case NC_BYTE: case NC_CHAR: case NC_UBYTE: return 1;
    case NC_SHORT: case NC_USHORT: return 2;
    case NC_INT: case NC_FLOAT: case NC_UINT: return 4;
    case NC_DOUBLE: case NC_INT64: case NC_UINT64: return 8;
    default: return 0;
    }
}

// ------------------------------------------------------------------ writer
struct Out {
    std::vector<unsigned char> b;
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void f64(double d) {
        uint64_t v;
        std::memcpy(&v, &d, 8);
        u64(v);
    }
    void name(const std::string &s) {
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        while (b.size() % 4) b.push_back(0);
    }
};

struct WAtt {
    std::string name;
    int type;  // NC_INT or NC_DOUBLE, one value
    double d;
    int i;
};
struct WVar {
    std::string name;
    std::vector<int> dims;  // C order
    std::vector<WAtt> atts;
    const double *data;     // host-order values, count = product of dims
    size_t count;
};

void put_atts(Out &o, const std::vector<WAtt> &atts) {
    if (atts.empty()) {
        o.u32(0);
        o.u32(0);
        return;
    }
    o.u32(TAG_ATT);
    o.u32((uint32_t)atts.size());
    for (const WAtt &a : atts) {
        o.name(a.name);
        o.u32((uint32_t)a.type);
        o.u32(1);
        if (a.type == NC_INT) o.u32((uint32_t)a.i);
        else o.f64(a.d);
    }
}

// header of a file with fixed-size dimensions, global attributes and double
// variables; `begin` holds the data offsets of the variables
Out header(int version, const std::vector<std::pair<std::string, size_t>> &dims, const std::vector<WAtt> &gatts,
           const std::vector<WVar> &vars, const std::vector<uint64_t> &begin) {
    Out o;
    o.b = {'C', 'D', 'F', (unsigned char)version};
    o.u32(0);  // numrecs
    o.u32(TAG_DIM);
    o.u32((uint32_t)dims.size());
    for (const auto &d : dims) {
        o.name(d.first);
        o.u32((uint32_t)d.second);
    }
    put_atts(o, gatts);
    o.u32(TAG_VAR);
    o.u32((uint32_t)vars.size());
    for (size_t v = 0; v < vars.size(); ++v) {
        const WVar &w = vars[v];
        o.name(w.name);
        o.u32((uint32_t)w.dims.size());
        for (int d : w.dims) o.u32((uint32_t)d);
        put_atts(o, w.atts);
        o.u32(NC_DOUBLE);
        const uint64_t vsize = (uint64_t)w.count * 8;
        o.u32(vsize > 0xFFFFFFFCull ? 0xFFFFFFFFu : (uint32_t)vsize);
        if (version == 1) o.u32((uint32_t)begin[v]);
        else o.u64(begin[v]);
    }
    return o;
}

int write_file(const char *path, const std::vector<std::pair<std::string, size_t>> &dims,
               const std::vector<WAtt> &gatts, const std::vector<WVar> &vars) {
    // the header's size does not depend on the offsets' values, only on
    // their width; the data follow it in variable order
    std::vector<uint64_t> begin(vars.size(), 0);
    int version = 1;
    for (int pass = 0; pass < 2; ++pass) {
        const size_t hsize = header(version, dims, gatts, vars, begin).b.size();
        uint64_t off = hsize;
        for (size_t v = 0; v < vars.size(); ++v) {
            begin[v] = off;
            off += (uint64_t)vars[v].count * 8;
        }
        if (version == 1 && off > (uint64_t)std::numeric_limits<int32_t>::max()) {
            version = 2;  // 64-bit offsets
            continue;
        }
        break;
    }
    Out o = header(version, dims, gatts, vars, begin);
    for (const WVar &w : vars)
        for (size_t i = 0; i < w.count; ++i) o.f64(w.data[i]);
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        pf_set_error("io_save_state: cannot create %s (%s)", path, std::strerror(errno));
        return PF_ERR_ARG;
    }
    const size_t n = std::fwrite(o.b.data(), 1, o.b.size(), f);
    const int c = std::fclose(f);
    if (n != o.b.size() || c != 0) {
        pf_set_error("io_save_state: write to %s failed", path);
        return PF_ERR_ARG;
    }
    return PF_OK;
}

// ------------------------------------------------------------------ reader
struct RAtt {
    std::string name;
    int type = 0;
    std::vector<double> v;  // numeric values (chars are not kept)
};
struct RVar {
    std::string name;
    std::vector<int> dims;
    std::vector<RAtt> atts;
    int type = 0;
    uint64_t begin = 0;
};
struct NcFile {
    int version = 0;
    std::vector<std::pair<std::string, uint64_t>> dims;
    std::vector<RAtt> gatts;
    std::vector<RVar> vars;
    std::vector<unsigned char> bytes;

    const RVar *var(const char *n) const {
        for (const RVar &v : vars)
            if (v.name == n) return &v;
        return nullptr;
    }
    static const RAtt *att(const std::vector<RAtt> &a, const char *n) {
        for (const RAtt &x : a)
            if (x.name == n && !x.v.empty()) return &x;
        return nullptr;
    }
};

struct In {
    const std::vector<unsigned char> &b;
    size_t p = 0;
    bool bad = false;
    explicit In(const std::vector<unsigned char> &x) : b(x) {}
    bool need(size_t n) {
        if (p + n > b.size()) bad = true;
        return !bad;
    }
    uint64_t be(int n) {
        if (!need(n)) return 0;
        uint64_t v = 0;
        for (int i = 0; i < n; ++i) v = (v << 8) | b[p++];
        return v;
    }
    uint32_t u32() { return (uint32_t)be(4); }
    uint64_t u64() { return be(8); }
    void pad() { p = (p + 3) & ~(size_t)3; }
};

double value_at(const unsigned char *q, int type) {
    uint64_t v = 0;
    const int n = type_size(type);
    for (int i = 0; i < n; ++i) v = (v << 8) | q[i];
    switch (type) {
    case NC_BYTE: return (double)(int8_t)v;
    case NC_UBYTE: return (double)(uint8_t)v;
    case NC_SHORT: return (double)(int16_t)v;
    case NC_USHORT: return (double)(uint16_t)v;
    case NC_INT: return (double)(int32_t)v;
    case NC_UINT: return (double)(uint32_t)v;
    case NC_INT64: return (double)(int64_t)v;
    case NC_UINT64: return (double)v;
    case NC_FLOAT: {
        uint32_t u = (uint32_t)v;
        float f;
        std::memcpy(&f, &u, 4);
        return f;
    }
    case NC_DOUBLE: {
        double d;
        std::memcpy(&d, &v, 8);
        return d;
    }
    default: return 0.0;
    }
}

bool read_atts(In &in, int nw, std::vector<RAtt> &out) {
    const uint32_t tag = in.u32();
    const uint64_t n = in.be(nw);
    if (tag == 0 && n == 0) return !in.bad;
    if (tag != TAG_ATT) return false;
    for (uint64_t i = 0; i < n && !in.bad; ++i) {
        RAtt a;
        const uint64_t ln = in.be(nw);
        if (!in.need(ln)) return false;
        a.name.assign((const char *)&in.b[in.p], ln);
        in.p += ln;
        in.pad();
        a.type = (int)in.u32();
        const uint64_t nv = in.be(nw);
        const int ts = type_size(a.type);
        if (ts == 0 || !in.need(nv * ts)) return false;
        if (a.type != NC_CHAR)
            for (uint64_t k = 0; k < nv; ++k) a.v.push_back(value_at(&in.b[in.p + k * ts], a.type));
        in.p += nv * ts;
        in.pad();
        out.push_back(a);
    }
    return !in.bad;
}

int read_file(const char *path, NcFile &nc) {
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        pf_set_error("io_load_state: state file not found!: %s", path);
        return PF_ERR_ARG;
    }
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    nc.bytes.resize(sz > 0 ? (size_t)sz : 0);
    const size_t got = nc.bytes.empty() ? 0 : std::fread(nc.bytes.data(), 1, nc.bytes.size(), f);
    std::fclose(f);
    if (got != nc.bytes.size() || got < 8 || std::memcmp(nc.bytes.data(), "CDF", 3) != 0) {
        pf_set_error("io_load_state: %s is not a netCDF-3 file", path);
        return PF_ERR_ARG;
    }
    nc.version = nc.bytes[3];
    if (nc.version != 1 && nc.version != 2 && nc.version != 5) {
        pf_set_error("io_load_state: %s: unsupported netCDF version %d", path, nc.version);
        return PF_ERR_ARG;
    }
    const int nw = nc.version == 5 ? 8 : 4;  // width of counts
    const int ow = nc.version == 1 ? 4 : 8;  // width of offsets
    In in(nc.bytes);
    in.p = 4;
    in.be(nw);  // numrecs
    bool ok = true;
    {
        const uint32_t tag = in.u32();
        const uint64_t n = in.be(nw);
        if (!(tag == 0 && n == 0)) {
            ok = tag == TAG_DIM;
            for (uint64_t i = 0; ok && i < n && !in.bad; ++i) {
                const uint64_t ln = in.be(nw);
                if (!in.need(ln)) break;
                std::string nm((const char *)&in.b[in.p], ln);
                in.p += ln;
                in.pad();
                nc.dims.push_back({nm, in.be(nw)});
            }
        }
    }
    ok = ok && read_atts(in, nw, nc.gatts);
    if (ok) {
        const uint32_t tag = in.u32();
        const uint64_t n = in.be(nw);
        if (!(tag == 0 && n == 0)) {
            ok = tag == TAG_VAR;
            for (uint64_t i = 0; ok && i < n && !in.bad; ++i) {
                RVar v;
                const uint64_t ln = in.be(nw);
                if (!in.need(ln)) break;
                v.name.assign((const char *)&in.b[in.p], ln);
                in.p += ln;
                in.pad();
                const uint64_t nd = in.be(nw);
                for (uint64_t d = 0; d < nd && !in.bad; ++d) v.dims.push_back((int)in.be(nw));
                ok = read_atts(in, nw, v.atts);
                v.type = (int)in.u32();
                in.be(nw);  // vsize
                v.begin = in.be(ow);
                nc.vars.push_back(v);
            }
        }
    }
    if (!ok || in.bad) {
        pf_set_error("io_load_state: %s: malformed netCDF header", path);
        return PF_ERR_ARG;
    }
    for (const RVar &v : nc.vars)
        for (int d : v.dims)
            if (d < 0 || d >= (int)nc.dims.size()) {
                pf_set_error("io_load_state: %s: variable %s has a bad dimension id", path, v.name.c_str());
                return PF_ERR_ARG;
            }
    return PF_OK;
}

// `count` values of variable v starting at element `start` (flattened C order)
int get_values(const NcFile &nc, const RVar &v, size_t start, size_t count, double *out) {
    const int ts = type_size(v.type);
    if (ts == 0 || v.type == NC_CHAR) {
        pf_set_error("io_load_coll: variable %s is not numeric", v.name.c_str());
        return PF_ERR_ARG;
    }
    for (int d : v.dims)
        if (nc.dims[d].second == 0) {
            pf_set_error("io_load_coll: record variable %s is not a state field", v.name.c_str());
            return PF_ERR_ARG;
        }
    const uint64_t a = v.begin + (uint64_t)start * ts, e = a + (uint64_t)count * ts;
    if (e > nc.bytes.size()) {
        pf_set_error("io_load_state: variable %s extends past the end of the file", v.name.c_str());
        return PF_ERR_ARG;
    }
    for (size_t i = 0; i < count; ++i) out[i] = value_at(&nc.bytes[a + i * ts], v.type);
    return PF_OK;
}

// ----------------------------------------------------- interpolation weights
// io_interp_wts (io.f90:232-262): for each output point the row of the
// inverse Taylor matrix over the (up to 2KL+1) nearest input points that
// gives the value at that point; io_interp (io.f90:268-288) applies it.
bool invert_small(int n, double *A) {  // row-major n x n, Gauss-Jordan with partial pivoting
    double I[(2 * KL + 1) * (2 * KL + 1)];
    for (int i = 0; i < n * n; ++i) I[i] = 0.0;
    for (int i = 0; i < n; ++i) I[i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
        if (A[p * n + c] == 0.0) return false;
        if (p != c)
            for (int k = 0; k < n; ++k) {
                std::swap(A[p * n + k], A[c * n + k]);
                std::swap(I[p * n + k], I[c * n + k]);
            }
        const double inv = 1.0 / A[c * n + c];
        for (int k = 0; k < n; ++k) {
            A[c * n + k] *= inv;
            I[c * n + k] *= inv;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = A[r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                A[r * n + k] -= f * A[c * n + k];
                I[r * n + k] -= f * I[c * n + k];
            }
        }
    }
    for (int i = 0; i < n * n; ++i) A[i] = I[i];
    return true;
}

struct Interp {
    std::vector<int> lo, nn;       // first input point (0-based) and count per output point
    std::vector<double> w;         // weights [n][2KL+1]
};

bool interp_wts(const std::vector<double> &xi, const double *xo, int no, Interp &W) {
    const int ni = (int)xi.size(), L = 2 * KL + 1;
    W.lo.assign(no, 0);
    W.nn.assign(no, 0);
    W.w.assign((size_t)no * L, 0.0);
    for (int n = 0; n < no; ++n) {
        int j = 0;
        while (xi[j] < xo[n] - 1e-8 && j < ni - 1) ++j;
        const int l = std::max(0, j - KL), r = std::min(j + KL, ni - 1), m = r - l + 1;
        double A[(2 * KL + 1) * (2 * KL + 1)];
        for (int i = 0; i < m; ++i) A[i * m] = 1.0;
        for (int c = 1; c < m; ++c)
            for (int i = 0; i < m; ++i) A[i * m + c] = A[i * m + c - 1] * (xi[l + i] - xo[n]) / (double)c;
        if (!invert_small(m, A)) return false;
        W.lo[n] = l;
        W.nn[n] = m;
        for (int i = 0; i < m; ++i) W.w[(size_t)n * L + i] = A[i];  // first row of the inverse
    }
    return true;
}

void interp_apply(const Interp &W, const double *fi, int no, double *fo) {
    const int L = 2 * KL + 1;
    for (int n = 0; n < no; ++n) {
        double s = 0.0;
        for (int i = 0; i < W.nn[n]; ++i) s += W.w[(size_t)n * L + i] * fi[W.lo[n] + i];
        fo[n] = s;
    }
}

int harmonics(int K, int M) { return (2 * K - 1) * M - (K - 1); }

}  // namespace

// ------------------------------------------------------------- host C ABI
extern "C" int pf_state_write(const char *path, int N, int K, int M, int Mp, const double *r, const double *ur_re,
                              const double *ur_im, const double *ut_re, const double *ut_im, const double *uz_re,
                              const double *uz_im, const double *scalars) {
    PF_ARG(path && r && ur_re && ur_im && ut_re && ut_im && uz_re && uz_im && scalars,
           "pf_state_write: null argument");
    PF_ARG(N > 0 && K > 0 && M > 0 && Mp > 0, "pf_state_write: bad size");
    const int H = harmonics(K, M);
    const size_t nf = (size_t)N * H;
    std::vector<double> fld[3];
    const double *src[3][2] = {{ur_re, ur_im}, {ut_re, ut_im}, {uz_re, uz_im}};
    for (int c = 0; c < 3; ++c) {
        fld[c].resize(2 * nf);
        std::memcpy(fld[c].data(), src[c][0], nf * sizeof(double));
        std::memcpy(fld[c].data() + nf, src[c][1], nf * sizeof(double));
    }
    const std::vector<std::pair<std::string, size_t>> dims = {{"r", (size_t)N}, {"H", (size_t)H}, {"ReIm", 2}};
    const std::vector<WAtt> g = {{"t", NC_DOUBLE, scalars[0], 0}, {"Re", NC_DOUBLE, scalars[1], 0},
                                 {"alpha", NC_DOUBLE, scalars[2], 0}};
    const std::vector<WAtt> km = {{"K", NC_INT, 0.0, K}, {"M", NC_INT, 0.0, M}, {"Mp", NC_INT, 0.0, Mp}};
    const std::vector<WVar> vars = {
        {"r", {0}, {}, r, (size_t)N},
        {"dt", {}, {}, &scalars[3], 1},
        {"dtcor", {}, {}, &scalars[4], 1},
        {"dtcfl", {}, {}, &scalars[5], 1},
        {"Ur", {2, 1, 0}, km, fld[0].data(), 2 * nf},
        {"Ut", {2, 1, 0}, km, fld[1].data(), 2 * nf},
        {"Uz", {2, 1, 0}, km, fld[2].data(), 2 * nf},
    };
    return write_file(path, dims, g, vars);
}

extern "C" int pf_state_read(const char *path, int N, int K, int M, int Mp, const double *r, double *ur_re,
                             double *ur_im, double *ut_re, double *ut_im, double *uz_re, double *uz_im,
                             double *scalars, int *changes) {
    PF_ARG(path && r && ur_re && ur_im && ut_re && ut_im && uz_re && uz_im && scalars,
           "pf_state_read: null argument");
    PF_ARG(N > 0 && K > 0 && M > 0 && Mp > 0, "pf_state_read: bad size");
    NcFile nc;
    PF_TRY(read_file(path, nc));
    const double nan = std::numeric_limits<double>::quiet_NaN();
    const char *gn[3] = {"t", "Re", "alpha"};
    for (int i = 0; i < 3; ++i) {
        const RAtt *a = NcFile::att(nc.gatts, gn[i]);
        scalars[i] = a ? a->v[0] : nan;
    }
    const char *sn[3] = {"dt", "dtcor", "dtcfl"};
    for (int i = 0; i < 3; ++i) {
        const RVar *v = nc.var(sn[i]);
        scalars[3 + i] = nan;
        if (v && v->dims.empty()) PF_TRY(get_values(nc, *v, 0, 1, &scalars[3 + i]));
    }
    int ch = 0;
    // radial points of the file, extended by KL mirrored points across the
    // axis (io.f90:131-140)
    int rd = -1;
    for (size_t d = 0; d < nc.dims.size(); ++d)
        if (nc.dims[d].first == "r") rd = (int)d;
    const RVar *rv = nc.var("r");
    if (rd < 0 || !rv || rv->dims.size() != 1) {
        pf_set_error("io_load_state: %s has no radial coordinate r", path);
        return PF_ERR_ARG;
    }
    const int N_ = (int)nc.dims[rd].second;
    std::vector<double> rx(KL + N_);
    PF_TRY(get_values(nc, *rv, 0, N_, rx.data() + KL));
    for (int i = 0; i < KL; ++i) rx[i] = (i < N_) ? -rx[2 * KL - 1 - i] : 0.0;  // r(1-KL:0) = -r(KL:1:-1)
    bool interp = N_ != N;
    if (!interp)
        for (int n = 0; n < N; ++n) interp = interp || std::fabs(r[n] - rx[KL + n]) > 1e-8;
    Interp W;
    if (interp) {
        if (N_ < KL) {
            pf_set_error("io_load_state: %s has %d radial points, fewer than KL", path, N_);
            return PF_ERR_ARG;
        }
        if (!interp_wts(rx, r, N, W)) {
            pf_set_error("matrix inversion error 1");
            return PF_ERR_SINGULAR;
        }
        ch |= 1;
    }
    const int H = harmonics(K, M);
    const char *fn[3] = {"Ur", "Ut", "Uz"};
    const int S[3] = {1, 1, 0};  // parity of the component across the axis
    double *dst[3][2] = {{ur_re, ur_im}, {ut_re, ut_im}, {uz_re, uz_im}};
    std::vector<double> f(KL + N_);
    for (int c = 0; c < 3; ++c) {
        const RVar *v = nc.var(fn[c]);
        if (!v) {
            pf_set_error("Field %s not found!", fn[c]);
            return PF_ERR_ARG;
        }
        const RAtt *aK = NcFile::att(v->atts, "K"), *aM = NcFile::att(v->atts, "M"), *aP = NcFile::att(v->atts, "Mp");
        if (!aK || !aM || !aP || v->dims.size() != 3 || nc.dims[v->dims[0]].second != 2 ||
            (int)nc.dims[v->dims[2]].second != N_) {
            pf_set_error("io_load_coll: %s is not a (ReIm, H, r) field with K, M, Mp", fn[c]);
            return PF_ERR_ARG;
        }
        const int K_ = (int)aK->v[0], M_ = (int)aM->v[0], Mp_ = (int)aP->v[0];
        const int H_ = (int)nc.dims[v->dims[1]].second;
        if (Mp_ != Mp && M_ > 2) {
            pf_set_error("io_load_coll: Mp /= i_Mp");
            return PF_ERR_ARG;
        }
        if (K_ != K) ch |= 2;
        if (M_ != M) ch |= 4;
        if (Mp_ != Mp) ch |= 8;
        for (int p = 0; p < 2; ++p) std::memset(dst[c][p], 0, sizeof(double) * (size_t)N * H);
        // the mode walk of io_load_coll (io.f90:196-226), file index counted
        // exactly as there
        const int K1 = std::max(K_, K) - 1, M1 = std::max(M_, M) - 1;
        int nh_f = -1, nh = -1;
        for (int m = 0; m <= M1; ++m)
            for (int k = -K1; k <= K1; ++k) {
                if (k < 0 && m == 0) continue;
                if (std::abs(k) >= K || m >= M) {
                    ++nh_f;
                    continue;
                }
                ++nh;
                if (std::abs(k) >= K_ || m >= M_) continue;
                ++nh_f;
                if (nh_f >= H_) continue;  // nf90_get_var fails there and leaves the mode zero
                for (int p = 0; p < 2; ++p) {
                    double *out = dst[c][p] + (size_t)nh * N;
                    const size_t start = ((size_t)p * H_ + nh_f) * N_;
                    if (interp) {
                        PF_TRY(get_values(nc, *v, start, N_, f.data() + KL));
                        const double sg = ((m * Mp + S[c]) % 2 == 1) ? -1.0 : 1.0;
                        for (int i = 0; i < KL; ++i) f[i] = sg * f[2 * KL - 1 - i];
                        interp_apply(W, f.data(), N, out);
                    } else {
                        PF_TRY(get_values(nc, *v, start, N_, out));
                    }
                }
            }
    }
    if (changes) *changes = ch;
    return PF_OK;
}

// ---------------------------------------------------------- context C ABI
extern "C" int pf_io_save_state(pf_ctx *ctx, const char *path) {
    PF_ARG(ctx && path, "pf_io_save_state: null argument");
    const Geo &g = ctx->g;
    const size_t nf = (size_t)g.N * g.H;
    std::vector<double> a(6 * nf);
    PF_TRY(pf_vel_get_state(ctx, &a[0], &a[nf], &a[2 * nf], &a[3 * nf], &a[4 * nf], &a[5 * nf]));
    const double sc[6] = {ctx->tim.t, ctx->cfg.Re, ctx->cfg.alpha, ctx->tim.dt, ctx->tim.corr_dt, ctx->tim.cfl_dt};
    return pf_state_write(path, g.N, g.K, g.M, g.Mp, ctx->hm.r.data(), &a[0], &a[nf], &a[2 * nf], &a[3 * nf],
                          &a[4 * nf], &a[5 * nf], sc);
}

extern "C" int pf_io_load_state(pf_ctx *ctx, const char *path, int flags, int *changes) {
    PF_ARG(ctx && path, "pf_io_load_state: null argument");
    const Geo &g = ctx->g;
    const size_t nf = (size_t)g.N * g.H;
    std::vector<double> a(6 * nf);
    double sc[6];
    PF_TRY(pf_state_read(path, g.N, g.K, g.M, g.Mp, ctx->hm.r.data(), &a[0], &a[nf], &a[2 * nf], &a[3 * nf],
                         &a[4 * nf], &a[5 * nf], sc, changes));
    if ((flags & PF_IO_TIME_FROM_FILE) && !std::isnan(sc[0])) ctx->tim.t = sc[0];
    if (ctx->cfg.dt < 0.0) {
        if (std::isnan(sc[3])) {
            pf_set_error("io_load_state: %s has no dt for an adaptive-dt run", path);
            return PF_ERR_ARG;
        }
        ctx->tim.dt = sc[3];
    } else {
        ctx->tim.dt = ctx->cfg.dt;
    }
    if (!std::isnan(sc[4])) ctx->tim.corr_dt = sc[4];
    if (!std::isnan(sc[5])) ctx->tim.cfl_dt = sc[5];
    return pf_vel_set_state(ctx, &a[0], &a[nf], &a[2 * nf], &a[3 * nf], &a[4 * nf], &a[5 * nf]);
}
