// The reference's NetCDF result file (Common/IO.h:136-276 OutputNetCDF3D_header,
// :340-377 OutputNetCDF3D_layer; called by FluidSolver3D.cpp:206 and :258), written
// without libnetcdf: the same dimensions, variables, attributes and values in a
// NetCDF classic file (64-bit offset format, "CDF\2") instead of the NetCDF-4 / HDF5
// container the reference asks libnetcdf for.  Host code only.
//
// Classic format, as published by Unidata: a header (magic, record count, the
// dimension, global attribute and variable lists; names and attribute values padded
// to 4 bytes; every number big-endian; each variable's size of one record and its
// begin offset), the fixed-size variables one after another, then the records, each
// holding one slab of every record variable in definition order.
#include "adi_b200.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

enum : uint32_t { NC_DIMENSION = 0x0A, NC_VARIABLE = 0x0B, NC_ATTRIBUTE = 0x0C };
enum : uint32_t { NC_CHAR = 2, NC_FLOAT = 5, NC_DOUBLE = 6 };
constexpr double FILL_DOUBLE = 9.9692099683868690e+36;   // NetCDF's default fill value for doubles
constexpr float MISSING = 99999.0f;                        // MISSING_VALUE, Common/Geometry.h:25

struct Buf {
    std::vector<unsigned char> b;
    void u32(uint32_t v)
    {
        for (int s = 24; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void u64(uint64_t v)
    {
        for (int s = 56; s >= 0; s -= 8) b.push_back((unsigned char)(v >> s));
    }
    void f32(float f)
    {
        uint32_t v;
        memcpy(&v, &f, 4);
        u32(v);
    }
    void f64(double d)
    {
        uint64_t v;
        memcpy(&v, &d, 8);
        u64(v);
    }
    void pad4()
    {
        while (b.size() % 4) b.push_back(0);
    }
    void name(const std::string &s)
    {
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        pad4();
    }
};

struct Att {
    std::string name;
    uint32_t type;
    std::string text;          // NC_CHAR
    std::vector<double> nums;  // NC_FLOAT / NC_DOUBLE
};

Att text(const char *n, const std::string &s) { return Att{n, NC_CHAR, s, {}}; }
Att nums(const char *n, uint32_t type, std::vector<double> v) { return Att{n, type, "", std::move(v)}; }

struct Var {
    std::string name;
    std::vector<uint32_t> dims;   // dimension ids
    std::vector<Att> atts;
    uint32_t type;
    uint64_t vsize = 0, begin = 0;
    bool record = false;
};

void put_atts(Buf &h, const std::vector<Att> &atts)
{
    if (atts.empty()) {
        h.u32(0);
        h.u32(0);
        return;
    }
    h.u32(NC_ATTRIBUTE);
    h.u32((uint32_t)atts.size());
    for (const Att &a : atts) {
        h.name(a.name);
        h.u32(a.type);
        if (a.type == NC_CHAR) {
            h.u32((uint32_t)a.text.size());
            h.b.insert(h.b.end(), a.text.begin(), a.text.end());
        } else {
            h.u32((uint32_t)a.nums.size());
            for (double v : a.nums) {
                if (a.type == NC_FLOAT) h.f32((float)v);
                else h.f64(v);
            }
        }
        h.pad4();
    }
}

// The variables of the reference's file, in its definition order (IO.h:160-172):
// x, y, z, time, then u, v, w, T (double, [t][x][y][z]) and d (float, [x][y]) when
// asked for; dimension ids x 0, y 1, z 2, t 3.
std::vector<Var> define_vars(const adi_bbox3d &bb, double time, int nx, int ny, int nz, const bool use[5],
                             bool xy_degree_units)
{
    static const char *shortn[5] = {"u", "v", "w", "T", "d"};
    static const char *longn[5] = {"x-velocity", "y-velocity", "z-velocity", "temperature", "depth"};
    std::vector<Var> vars;
    // attributes in the order the reference puts them (IO.h:174-228)
    Var x{"x", {0}, {}, NC_FLOAT}, y{"y", {1}, {}, NC_FLOAT}, z{"z", {2}, {}, NC_FLOAT}, t{"time", {3}, {}, NC_DOUBLE};
    x.atts = {nums("actual_range", NC_FLOAT, {bb.pmin[0], bb.pmax[0]}), text("long_name", "x coord"),
              text("units", xy_degree_units ? "degree_north" : "metres")};
    y.atts = {nums("actual_range", NC_FLOAT, {bb.pmin[1], bb.pmax[1]}), text("long_name", "y coord"),
              text("units", xy_degree_units ? "degree_east" : "metres")};
    z.atts = {text("units", "metres"), nums("actual_range", NC_FLOAT, {bb.pmin[2], bb.pmax[2]}),
              text("long_name", "z coord")};
    t.atts = {text("units", "s"), nums("actual_range", NC_DOUBLE, {0.0, time}), text("long_name", "time")};
    t.record = true;
    vars = {x, y, z, t};
    for (int i = 0; i < 5; i++) {
        if (!use[i]) continue;
        Var v;
        v.name = shortn[i];
        if (i == 4) {
            v.dims = {0, 1};
            v.type = NC_FLOAT;
        } else {
            v.dims = {3, 0, 1, 2};
            v.type = NC_DOUBLE;
            v.record = true;
        }
        const char *units = shortn[i][0] == 'T' ? "tmp" : (shortn[i][0] == 'd' ? "m" : "m/s");
        v.atts = {text("units", units), nums("actual_range", NC_DOUBLE, {-1.0, 1.0}),
                  nums("valid_range", NC_DOUBLE, {-1.0, 1.0}), nums("missing_value", NC_FLOAT, {MISSING}),
                  text("long_name", longn[i]), text("var_desc", shortn[i])};
        vars.push_back(v);
    }
    const uint64_t dimlen[3] = {(uint64_t)nx, (uint64_t)ny, (uint64_t)nz};
    for (Var &v : vars) {
        uint64_t n = v.type == NC_DOUBLE ? 8 : 4;
        for (uint32_t dd : v.dims)
            if (dd != 3) n *= dimlen[dd];
        v.vsize = (n + 3) / 4 * 4;
    }
    return vars;
}

std::vector<unsigned char> header_bytes(const std::vector<Var> &vars, uint32_t numrecs, int nx, int ny, int nz)
{
    Buf h;
    h.b = {'C', 'D', 'F', 2};
    h.u32(numrecs);
    h.u32(NC_DIMENSION);
    h.u32(4);
    h.name("x"); h.u32((uint32_t)nx);
    h.name("y"); h.u32((uint32_t)ny);
    h.name("z"); h.u32((uint32_t)nz);
    h.name("t"); h.u32(0);   // the record (unlimited) dimension
    put_atts(h, {text("Conventions", "COARDS"), text("title", "cmc-fluid-solver results"),
                 text("history", "created by using cmc-fluid-solver"), text("description", "Test data"),
                 text("platform", "Model")});
    h.u32(NC_VARIABLE);
    h.u32((uint32_t)vars.size());
    for (const Var &v : vars) {
        h.name(v.name);
        h.u32((uint32_t)v.dims.size());
        for (uint32_t d : v.dims) h.u32(d);
        put_atts(h, v.atts);
        h.u32(v.type);
        h.u32((uint32_t)v.vsize);
        h.u64(v.begin);
    }
    return h.b;
}

struct Layout {
    std::vector<Var> vars;
    uint64_t header = 0, recs_begin = 0, recsize = 0;
};

// Begin offsets: the header, the fixed-size variables in order, then the records.
void place(Layout &L, uint32_t numrecs, int nx, int ny, int nz)
{
    L.header = header_bytes(L.vars, numrecs, nx, ny, nz).size();   // begins do not change its size
    uint64_t off = L.header;
    for (Var &v : L.vars)
        if (!v.record) {
            v.begin = off;
            off += v.vsize;
        }
    L.recs_begin = off;
    L.recsize = 0;
    for (Var &v : L.vars)
        if (v.record) {
            v.begin = off + L.recsize;
            L.recsize += v.vsize;
        }
}

bool parse_vars(const char *list, bool use[5])
{
    static const char *shortn[5] = {"u", "v", "w", "T", "d"};
    for (int i = 0; i < 5; i++) use[i] = false;
    if (!list) return false;
    std::string s(list);
    size_t p = 0;
    while (p <= s.size()) {
        size_t q = s.find(',', p);
        if (q == std::string::npos) q = s.size();
        const std::string tok = s.substr(p, q - p);
        for (int i = 0; i < 5; i++)
            if (tok == shortn[i]) use[i] = true;
        p = q + 1;
    }
    return true;
}

bool write_at(FILE *f, uint64_t off, const void *p, size_t n)
{
    if (fseeko(f, (off_t)off, SEEK_SET) != 0) return false;
    return fwrite(p, 1, n, f) == n;
}

std::vector<unsigned char> be_doubles(const double *v, size_t n)
{
    Buf b;
    b.b.reserve(n * 8);
    for (size_t i = 0; i < n; i++) b.f64(v[i]);
    return b.b;
}

// The header's variable list, read back from a file this writer made.
bool read_layout(FILE *f, Layout &L, uint32_t &numrecs, int dims[3])
{
    auto rd32 = [&](uint32_t &v) {
        unsigned char c[4];
        if (fread(c, 1, 4, f) != 4) return false;
        v = (uint32_t)c[0] << 24 | (uint32_t)c[1] << 16 | (uint32_t)c[2] << 8 | c[3];
        return true;
    };
    auto rd64 = [&](uint64_t &v) {
        uint32_t a, b;
        if (!rd32(a) || !rd32(b)) return false;
        v = (uint64_t)a << 32 | b;
        return true;
    };
    auto rdname = [&](std::string &s) {
        uint32_t n;
        if (!rd32(n) || n > 256) return false;
        const uint32_t padded = (n + 3) / 4 * 4;
        std::vector<char> c(padded);
        if (fread(c.data(), 1, padded, f) != padded) return false;
        s.assign(c.data(), n);
        return true;
    };
    auto skip_atts = [&]() {
        uint32_t tag, n;
        if (!rd32(tag) || !rd32(n)) return false;
        for (uint32_t a = 0; a < n; a++) {
            std::string nm;
            uint32_t type, cnt;
            if (!rdname(nm) || !rd32(type) || !rd32(cnt)) return false;
            const uint32_t sz = type == NC_CHAR ? 1 : (type == NC_FLOAT ? 4 : 8);
            if (fseeko(f, (off_t)((cnt * sz + 3) / 4 * 4), SEEK_CUR) != 0) return false;
        }
        return true;
    };
    unsigned char magic[4];
    if (fseeko(f, 0, SEEK_SET) != 0 || fread(magic, 1, 4, f) != 4) return false;
    if (memcmp(magic, "CDF\2", 4) != 0) return false;
    uint32_t tag, n;
    if (!rd32(numrecs) || !rd32(tag) || !rd32(n) || tag != NC_DIMENSION || n != 4) return false;
    for (int d = 0; d < 4; d++) {
        std::string nm;
        uint32_t len;
        if (!rdname(nm) || !rd32(len)) return false;
        if (d < 3) dims[d] = (int)len;
    }
    if (!skip_atts()) return false;
    if (!rd32(tag) || !rd32(n) || tag != NC_VARIABLE) return false;
    L.vars.clear();
    for (uint32_t i = 0; i < n; i++) {
        Var v;
        uint32_t nd;
        if (!rdname(v.name) || !rd32(nd) || nd > 4) return false;
        v.dims.resize(nd);
        for (uint32_t &d : v.dims)
            if (!rd32(d)) return false;
        if (!skip_atts()) return false;
        uint32_t vs;
        if (!rd32(v.type) || !rd32(vs) || !rd64(v.begin)) return false;
        v.vsize = vs;
        v.record = !v.dims.empty() && v.dims[0] == 3;
        L.vars.push_back(v);
    }
    L.header = (uint64_t)ftello(f);
    L.recsize = 0;
    L.recs_begin = UINT64_MAX;
    for (const Var &v : L.vars)
        if (v.record) {
            L.recsize += v.vsize;
            if (v.begin < L.recs_begin) L.recs_begin = v.begin;
        }
    return true;
}

// Fills records [from, to) with fill values (time and the data variables).
bool fill_records(FILE *f, const Layout &L, uint32_t from, uint32_t to)
{
    std::vector<unsigned char> fill;
    for (uint32_t r = from; r < to; r++)
        for (const Var &v : L.vars) {
            if (!v.record) continue;
            if (fill.size() != v.vsize) {
                fill.clear();
                Buf b;
                for (uint64_t k = 0; k < v.vsize / 8; k++) b.f64(FILL_DOUBLE);
                fill = b.b;
            }
            if (!write_at(f, v.begin + (uint64_t)r * L.recsize, fill.data(), fill.size())) return false;
        }
    return true;
}

} // namespace

extern "C" {

adi_status adi_nc_write_header(const char *path, const adi_bbox3d *bbox, const float *depth, int depth_nx,
                               int depth_ny, double timestep, double time, int outdimx, int outdimy, int outdimz,
                               const char *vars, int xy_degree_units)
{
    bool use[5];
    if (!path || !bbox || !parse_vars(vars, use) || outdimx < 1 || outdimy < 1 || outdimz < 1 || !(timestep > 0) ||
        !(time >= 0) || time / timestep > 1e7)
        return ADI_ERR_BAD_ARG;
    if (use[4] && (!depth || depth_nx < 1 || depth_ny < 1)) return ADI_ERR_BAD_ARG;
    Layout L;
    L.vars = define_vars(*bbox, time, outdimx, outdimy, outdimz, use, xy_degree_units != 0);
    // the 64-bit offset format stores a variable's size (one record of it) in 32 bits
    for (const Var &v : L.vars)
        if (v.vsize > 0xFFFFFFFCull) return ADI_ERR_BAD_ARG;
    // the time axis is written for time / timestep records (IO.h:260-266)
    const uint32_t count = (uint32_t)(int)(time / timestep);
    place(L, count, outdimx, outdimy, outdimz);
    FILE *f = fopen(path, "wb");
    if (!f) return ADI_ERR_BAD_ARG;
    bool ok = true;
    const std::vector<unsigned char> hdr = header_bytes(L.vars, count, outdimx, outdimy, outdimz);
    ok = ok && write_at(f, 0, hdr.data(), hdr.size());
    // axes (IO.h:234-258): value = pMin + (float)((pMax - pMin) / n) * i, in FTYPE = float
    const int n3[3] = {outdimx, outdimy, outdimz};
    for (int a = 0; a < 3 && ok; a++) {
        const float dd = (float)(bbox->pmax[a] - bbox->pmin[a]) / (n3[a]);
        Buf b;
        for (int i = 0; i < n3[a]; i++) b.f32(bbox->pmin[a] + dd * i);
        b.pad4();
        ok = write_at(f, L.vars[a].begin, b.b.data(), b.b.size());
    }
    // depths at the output resolution (DepthInfo3D's point sampling, Common/Geometry.h:429-441)
    for (const Var &v : L.vars)
        if (ok && v.name == "d") {
            Buf b;
            for (int i = 0; i < outdimx; i++)
                for (int j = 0; j < outdimy; j++) {
                    const int x = i * depth_nx / outdimx, y = j * depth_ny / outdimy;
                    b.f32(depth[y + depth_ny * x]);
                }
            ok = write_at(f, v.begin, b.b.data(), b.b.size());
        }
    // every record allocated by the time axis: fill values, then the time values
    ok = ok && fill_records(f, L, 0, count);
    for (uint32_t r = 0; r < count && ok; r++) {
        const double tv = r * timestep;
        const std::vector<unsigned char> b = be_doubles(&tv, 1);
        ok = write_at(f, L.vars[3].begin + (uint64_t)r * L.recsize, b.data(), b.size());
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? ADI_OK : ADI_ERR_BAD_ARG;
}

adi_status adi_nc_write_layer(const char *path, const void *vel, int vel_elem_bytes, const double *T, int layer,
                              int outdimx, int outdimy, int outdimz, const char *vars)
{
    bool use[5];
    if (!path || !vel || !T || layer < 0 || !parse_vars(vars, use) || (vel_elem_bytes != 4 && vel_elem_bytes != 8))
        return ADI_ERR_BAD_ARG;
    FILE *f = fopen(path, "r+b");
    if (!f) return ADI_ERR_BAD_ARG;
    Layout L;
    uint32_t numrecs = 0;
    int dims[3] = {0, 0, 0};
    bool ok = read_layout(f, L, numrecs, dims) && dims[0] == outdimx && dims[1] == outdimy && dims[2] == outdimz;
    if (ok && (uint32_t)layer >= numrecs) {
        // a layer past the written records extends the record count (its time stays the fill value)
        ok = fill_records(f, L, numrecs, (uint32_t)layer + 1);
        numrecs = (uint32_t)layer + 1;
        Buf b;
        b.u32(numrecs);
        ok = ok && write_at(f, 4, b.b.data(), 4);
    }
    const size_t n = (size_t)outdimx * outdimy * outdimz;
    std::vector<double> vals(n);
    for (const Var &v : L.vars) {
        if (!ok) break;
        if (!v.record || v.name == "time" || v.name.size() != 1) continue;
        const char c = v.name[0];
        int comp = c == 'u' ? 0 : (c == 'v' ? 1 : (c == 'w' ? 2 : 3));
        if (!use[c == 'T' ? 3 : comp]) continue;   // only the variables asked for (IO.h:352-356)
        for (size_t idx = 0; idx < n; idx++) {
            if (comp == 3) vals[idx] = T[idx];
            else if (vel_elem_bytes == 4) vals[idx] = ((const float *)vel)[3 * idx + comp];
            else vals[idx] = ((const double *)vel)[3 * idx + comp];
        }
        const std::vector<unsigned char> b = be_doubles(vals.data(), n);
        ok = write_at(f, v.begin + (uint64_t)layer * L.recsize, b.data(), b.size());
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? ADI_OK : ADI_ERR_BAD_ARG;
}

} // extern "C"
