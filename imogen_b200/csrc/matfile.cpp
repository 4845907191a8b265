// MAT-file Level 5 slice files of save/resultsHandler.m:26-113, and their reader for resuming a run
// (experiment/Initializer.m:269-292, loadDataFromFile).
//
// Writer: one struct variable sx_<label>_<suffix> whose fields are those resultsHandler assigns, in
// its order: gamma, time (TimeManager.toStruct: time, history, iterMax, timeMax, wallMax, started,
// iteration), about, ver, iter, [tread (TreadmillManager.toStruct: direction, history)], mass, momX,
// momY, momZ, ener, magX, magY, magZ (empty without the magnet), grav (empty: no gravity on this path),
// dGrid (1x3 cell) and dim.  The arrays are SaveManager.getSaveSlice cuts (squeezed as MATLAB's
// squeeze does), FP64, column-major (x fastest, as the state is held).  Elements are written
// uncompressed (MATLAB reads either form).
//
// Reader: little-endian Level 5 files, uncompressed or with miCOMPRESSED (zlib) elements as MATLAB 7
// writes by default; numeric data stored in any MAT numeric type (MATLAB narrows integer-valued doubles)
// is widened to double.  Sparse, complex and object arrays are not read.  Like loadDataFromFile it takes
// the first variable of the file and its mass, ener, momX/Y/Z and magX/Y/Z fields (B zero when empty).
#include <zlib.h>

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "imogen_b200.h"

namespace {

enum MiType {
    miINT8 = 1, miUINT8 = 2, miINT16 = 3, miUINT16 = 4, miINT32 = 5, miUINT32 = 6, miSINGLE = 7, miDOUBLE = 9,
    miINT64 = 12, miUINT64 = 13, miMATRIX = 14, miCOMPRESSED = 15, miUTF8 = 16, miUTF16 = 17, miUTF32 = 18
};
enum MxClass {
    mxCELL = 1, mxSTRUCT = 2, mxOBJECT = 3, mxCHAR = 4, mxSPARSE = 5, mxDOUBLE = 6, mxSINGLE = 7, mxINT8 = 8,
    mxUINT8 = 9, mxINT16 = 10, mxUINT16 = 11, mxINT32 = 12, mxUINT32 = 13, mxINT64 = 14, mxUINT64 = 15
};

// One MATLAB value: numeric (as double), char, 1x1 struct or cell.
struct Node {
    int cls = mxDOUBLE;
    std::vector<int> dims{0, 0};
    std::vector<double> num;
    std::string text;
    std::vector<std::string> fnames;
    std::vector<Node> fields;
    std::vector<Node> cells;
};

Node num_node(std::vector<int> dims, std::vector<double> v) {
    Node n;
    n.dims = std::move(dims);
    n.num = std::move(v);
    return n;
}
Node scalar(double v) { return num_node({1, 1}, {v}); }
Node empty() { return num_node({0, 0}, {}); }
Node text(const std::string& s) {
    Node n;
    n.cls = mxCHAR;
    n.dims = {1, (int)s.size()};
    if (s.empty()) n.dims = {0, 0};
    n.text = s;
    return n;
}
Node strct(std::vector<std::pair<std::string, Node>> f) {
    Node n;
    n.cls = mxSTRUCT;
    n.dims = {1, 1};
    for (auto& p : f) {
        n.fnames.push_back(p.first);
        n.fields.push_back(std::move(p.second));
    }
    return n;
}

// ---- writer -----------------------------------------------------------------------------------------
struct Out {
    std::vector<uint8_t> b;
    void raw(const void* p, size_t n) { b.insert(b.end(), (const uint8_t*)p, (const uint8_t*)p + n); }
    void u32(uint32_t v) { raw(&v, 4); }
    void pad8() { while (b.size() % 8) b.push_back(0); }
    void element(uint32_t type, const void* p, size_t n) {
        u32(type);
        u32((uint32_t)n);
        raw(p, n);
        pad8();
    }
};

void write_matrix(Out& o, const Node& n, const std::string& name);

void write_body(Out& o, const Node& n, const std::string& name) {
    const uint32_t flags[2] = {(uint32_t)n.cls, 0u};
    o.element(miUINT32, flags, 8);
    std::vector<int32_t> dims(n.dims.begin(), n.dims.end());
    o.element(miINT32, dims.data(), dims.size() * 4);
    o.element(miINT8, name.data(), name.size());
    switch (n.cls) {
        case mxCHAR: {
            std::vector<uint16_t> u(n.text.begin(), n.text.end());
            o.element(miUINT16, u.data(), u.size() * 2);
            break;
        }
        case mxSTRUCT: {
            size_t len = 1;
            for (const auto& f : n.fnames) len = std::max(len, f.size() + 1);
            const uint32_t small[2] = {(4u << 16) | miINT32, (uint32_t)len};   // field name length, small form
            o.raw(small, 8);
            std::vector<char> names(len * n.fnames.size(), 0);
            for (size_t i = 0; i < n.fnames.size(); ++i) std::memcpy(&names[i * len], n.fnames[i].data(), n.fnames[i].size());
            o.element(miINT8, names.data(), names.size());
            for (const auto& f : n.fields) write_matrix(o, f, "");
            break;
        }
        case mxCELL:
            for (const auto& c : n.cells) write_matrix(o, c, "");
            break;
        default:
            o.element(miDOUBLE, n.num.data(), n.num.size() * 8);
    }
}

void write_matrix(Out& o, const Node& n, const std::string& name) {
    Out body;
    write_body(body, n, name);
    o.u32(miMATRIX);
    o.u32((uint32_t)body.b.size());
    o.raw(body.b.data(), body.b.size());
}

// ---- reader -----------------------------------------------------------------------------------------
struct In {
    const uint8_t* p;
    size_t n;
    size_t at = 0;
    bool ok = true;
};

// One data element: type, payload bytes, and the offset after it (8-byte padded, small elements in 8).
bool next_element(In& in, uint32_t& type, std::vector<uint8_t>& data) {
    if (in.at + 8 > in.n) return false;
    uint32_t w0, w1;
    std::memcpy(&w0, in.p + in.at, 4);
    std::memcpy(&w1, in.p + in.at + 4, 4);
    if (w0 >> 16) {   // small data element: size in the upper half, data in the second word
        type = w0 & 0xffff;
        const uint32_t sz = w0 >> 16;
        if (sz > 4) return false;
        data.assign(in.p + in.at + 4, in.p + in.at + 4 + sz);
        in.at += 8;
        return true;
    }
    type = w0;
    const size_t sz = w1;
    if (in.at + 8 + sz > in.n) return false;
    data.assign(in.p + in.at + 8, in.p + in.at + 8 + sz);
    in.at += 8 + sz;
    if (type != miCOMPRESSED) in.at = (in.at + 7) & ~(size_t)7;
    if (in.at > in.n) in.at = in.n;
    return true;
}

bool to_doubles(uint32_t type, const std::vector<uint8_t>& d, std::vector<double>& out) {
    auto conv = [&](auto tag) {
        using V = decltype(tag);
        const size_t k = d.size() / sizeof(V);
        out.resize(k);
        for (size_t i = 0; i < k; ++i) {
            V v;
            std::memcpy(&v, d.data() + i * sizeof(V), sizeof(V));
            out[i] = (double)v;
        }
        return true;
    };
    switch (type) {
        case miINT8: return conv(int8_t());
        case miUINT8: return conv(uint8_t());
        case miINT16: return conv(int16_t());
        case miUINT16: return conv(uint16_t());
        case miINT32: return conv(int32_t());
        case miUINT32: return conv(uint32_t());
        case miSINGLE: return conv(float());
        case miDOUBLE: return conv(double());
        case miINT64: return conv(int64_t());
        case miUINT64: return conv(uint64_t());
        default: return false;
    }
}

bool inflate_all(const std::vector<uint8_t>& src, std::vector<uint8_t>& dst) {
    z_stream z{};
    if (inflateInit(&z) != Z_OK) return false;
    z.next_in = const_cast<Bytef*>(src.data());
    z.avail_in = (uInt)src.size();
    dst.clear();
    std::vector<uint8_t> buf(1 << 16);
    int r;
    do {
        z.next_out = buf.data();
        z.avail_out = (uInt)buf.size();
        r = inflate(&z, Z_NO_FLUSH);
        if (r != Z_OK && r != Z_STREAM_END) {
            inflateEnd(&z);
            return false;
        }
        dst.insert(dst.end(), buf.data(), buf.data() + (buf.size() - z.avail_out));
    } while (r != Z_STREAM_END && (z.avail_in > 0 || z.avail_out == 0));
    inflateEnd(&z);
    return r == Z_STREAM_END;
}

bool parse_matrix(const std::vector<uint8_t>& body, Node& n, std::string& name);

// The value of one top-level or nested element (miMATRIX, or miCOMPRESSED around one).
bool parse_value(uint32_t type, const std::vector<uint8_t>& data, Node& n, std::string& name) {
    if (type == miCOMPRESSED) {
        std::vector<uint8_t> raw;
        if (!inflate_all(data, raw)) return false;
        In in{raw.data(), raw.size()};
        uint32_t t2;
        std::vector<uint8_t> d2;
        if (!next_element(in, t2, d2)) return false;
        return parse_value(t2, d2, n, name);
    }
    if (type != miMATRIX) return false;
    return parse_matrix(data, n, name);
}

bool parse_matrix(const std::vector<uint8_t>& body, Node& n, std::string& name) {
    In in{body.data(), body.size()};
    uint32_t t;
    std::vector<uint8_t> d;
    if (body.empty()) {   // an empty miMATRIX: []
        n = empty();
        name.clear();
        return true;
    }
    if (!next_element(in, t, d) || d.size() < 8) return false;
    uint32_t flags;
    std::memcpy(&flags, d.data(), 4);
    n.cls = (int)(flags & 0xff);
    const bool complex = (flags >> 11) & 1;
    if (!next_element(in, t, d)) return false;
    std::vector<double> dv;
    if (!to_doubles(t, d, dv)) return false;
    n.dims.assign(dv.begin(), dv.end());
    if (!next_element(in, t, d)) return false;
    name.assign(d.begin(), d.end());
    size_t count = 1;
    for (int v : n.dims) count *= (size_t)v;
    switch (n.cls) {
        case mxCHAR: {
            if (count == 0) return true;
            if (!next_element(in, t, d)) return false;
            std::vector<double> c;
            if (t == miUTF8) c.assign(d.begin(), d.end());
            else if (t == miUTF16) { if (!to_doubles(miUINT16, d, c)) return false; }
            else if (!to_doubles(t, d, c)) return false;
            n.text.clear();
            for (double v : c) n.text.push_back((char)(int)v);
            return true;
        }
        case mxSTRUCT: {
            if (!next_element(in, t, d) || d.size() < 4) return false;
            int32_t len;
            std::memcpy(&len, d.data(), 4);
            if (!next_element(in, t, d) || len <= 0) return false;
            const size_t nf = d.size() / (size_t)len;
            for (size_t i = 0; i < nf; ++i) {
                const char* s = (const char*)d.data() + i * len;
                n.fnames.emplace_back(s, strnlen(s, (size_t)len));
            }
            n.fields.resize(nf * count);   // count elements of the struct array, fields in order each
            for (auto& f : n.fields) {
                std::string nm;
                if (!next_element(in, t, d) || !parse_value(t, d, f, nm)) return false;
            }
            return true;
        }
        case mxCELL: {
            n.cells.resize(count);
            for (auto& c : n.cells) {
                std::string nm;
                if (!next_element(in, t, d) || !parse_value(t, d, c, nm)) return false;
            }
            return true;
        }
        case mxDOUBLE: case mxSINGLE: case mxINT8: case mxUINT8: case mxINT16: case mxUINT16: case mxINT32:
        case mxUINT32: case mxINT64: case mxUINT64: {
            if (complex) return false;
            if (count == 0) {
                n.num.clear();
                return true;
            }
            if (!next_element(in, t, d) || !to_doubles(t, d, n.num)) return false;
            return n.num.size() == count;
        }
        default:
            return false;   // sparse, object, function handle
    }
}

const Node* field(const Node& s, const char* name) {
    if (s.cls != mxSTRUCT) return nullptr;
    for (size_t i = 0; i < s.fnames.size() && i < s.fields.size(); ++i)
        if (s.fnames[i] == name) return &s.fields[i];
    return nullptr;
}

thread_local std::string g_mat_err;
int mat_fail(int code, const std::string& why) {
    g_mat_err = why;
    return code;
}

// MATLAB squeeze of an array of size d (trailing singletons dropped, at least 2-D).
std::vector<int> squeezed(std::vector<int> d) {
    while (d.size() > 2 && d.back() == 1) d.pop_back();
    if (d.size() == 2) return d;
    std::vector<int> r;
    for (int v : d)
        if (v != 1) r.push_back(v);
    while (r.size() < 2) r.push_back(1);
    return r;
}

// SaveManager.getSaveSlice(array, type) (save/SaveManager.m:230-253) of a column-major grid array.
Node cut(const double* a, const int g[3], int type, const int idx[3]) {
    int lo[3] = {0, 0, 0}, hi[3] = {g[0], g[1], g[2]};
    auto fix = [&](int d) {
        lo[d] = idx[d] - 1;
        hi[d] = idx[d];
    };
    switch (type) {
        case 1: fix(1); fix(2); break;
        case 2: fix(0); fix(2); break;
        case 3: fix(0); fix(1); break;
        case 4: fix(2); break;
        case 5: fix(1); break;
        case 6: fix(0); break;
        default: break;
    }
    std::vector<double> v;
    v.reserve((size_t)(hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]));
    for (int z = lo[2]; z < hi[2]; ++z)
        for (int y = lo[1]; y < hi[1]; ++y)
            for (int x = lo[0]; x < hi[0]; ++x) v.push_back(a[x + (long long)g[0] * (y + (long long)g[1] * z)]);
    return num_node(squeezed({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]}), std::move(v));
}

const char* kLabels[8] = {"X", "Y", "Z", "XY", "XZ", "YZ", "XYZ", "SP-XYZ"};   // SaveManager.SLICELABELS
const char* kDims[8] = {"1D", "1D", "1D", "2D", "2D", "2D", "3D", "Cust"};

// genvarname: characters outside [A-Za-z0-9_] become their hex code 0xNN.
std::string valid_name(const std::string& s) {
    std::string r;
    for (unsigned char c : s) {
        if (std::isalnum(c) || c == '_') r.push_back((char)c);
        else {
            char h[8];
            std::snprintf(h, sizeof h, "0x%02X", c);
            r += h;
        }
    }
    if (r.empty() || !std::isalpha((unsigned char)r[0])) r = "x" + r;
    return r.substr(0, 63);
}

}  // namespace

extern "C" {

const char* img_slice_last_error(void) { return g_mat_err.c_str(); }

int img_slice_write(const char* path, const img_slice_meta* m, const img_slice_state* st) {
    if (!path || !m || !st || !st->mass || !st->mom || !st->ener) return mat_fail(IMG_ERR_ARG, "null argument");
    if (m->type < 1 || m->type > 8) return mat_fail(IMG_ERR_ARG, "slice type must be 1-8");
    const int* g = st->grid;
    for (int d = 0; d < 3; ++d) {
        if (g[d] < 1) return mat_fail(IMG_ERR_ARG, "grid extents must be >= 1");
        if (m->type <= 6 && (m->index[d] < 1 || m->index[d] > g[d]))
            return mat_fail(IMG_ERR_ARG, "slice index outside the grid");
    }
    const long long n = (long long)g[0] * g[1] * g[2];
    std::vector<double> hist(st->dt_history ? st->dt_history : nullptr,
                             st->dt_history ? st->dt_history + std::max(0, st->n_history) : nullptr);
    Node time = strct({{"time", scalar(st->time)},
                       {"history", num_node({(int)hist.size(), 1}, hist)},
                       {"iterMax", scalar(st->iter_max)},
                       {"timeMax", scalar(st->time_max)},
                       {"wallMax", scalar(m->wall_max)},
                       {"started", text(m->started ? m->started : "")},
                       {"iteration", scalar(st->iteration)}});
    std::vector<std::pair<std::string, Node>> f = {{"gamma", scalar(st->gamma)},
                                                   {"time", time},
                                                   {"about", text(m->about ? m->about : "")},
                                                   {"ver", scalar(m->version)},
                                                   {"iter", scalar(st->iteration)}};
    if (st->treadmill > 0) {   // TreadmillManager.toStruct: history(1:max(index-1, 1)), zeros preallocated
        std::vector<double> th;
        for (int i = 0; i < st->n_tread; ++i) th.push_back(st->tread_history[i]);
        if (th.empty()) th.push_back(0.0);
        f.push_back({"tread", strct({{"direction", scalar(st->treadmill)},
                                     {"history", num_node({(int)th.size(), 1}, th)}})});
    }
    const int t = m->type;
    f.push_back({"mass", cut(st->mass, g, t, m->index)});
    f.push_back({"momX", cut(st->mom, g, t, m->index)});
    f.push_back({"momY", cut(st->mom + n, g, t, m->index)});
    f.push_back({"momZ", cut(st->mom + 2 * n, g, t, m->index)});
    f.push_back({"ener", cut(st->ener, g, t, m->index)});
    const bool mag = st->magnet_active && st->mag;
    f.push_back({"magX", mag ? cut(st->mag, g, t, m->index) : empty()});
    f.push_back({"magY", mag ? cut(st->mag + n, g, t, m->index) : empty()});
    f.push_back({"magZ", mag ? cut(st->mag + 2 * n, g, t, m->index) : empty()});
    f.push_back({"grav", empty()});
    Node dg;
    dg.cls = mxCELL;
    dg.dims = {1, 3};
    for (int d = 0; d < 3; ++d) dg.cells.push_back(scalar(st->dgrid[d]));
    f.push_back({"dGrid", dg});
    f.push_back({"dim", text(kDims[t - 1])});
    const std::string var = valid_name(std::string("sx_") + kLabels[t - 1] + "_" + (m->suffix ? m->suffix : "FINAL"));

    Out o;
    char head[116];
    std::memset(head, ' ', sizeof head);
    const std::time_t now = std::time(nullptr);
    char date[64];
    std::strftime(date, sizeof date, "%a %b %d %H:%M:%S %Y", std::gmtime(&now));
    const std::string txt = std::string("MATLAB 5.0 MAT-file, Platform: GLNXA64, Created on: ") + date;
    std::memcpy(head, txt.data(), std::min(txt.size(), sizeof head));
    o.raw(head, sizeof head);
    const uint8_t subsys[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    o.raw(subsys, 8);
    const uint16_t ver = 0x0100;
    o.raw(&ver, 2);
    o.raw("IM", 2);
    write_matrix(o, strct(f), var);
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return mat_fail(IMG_ERR_ARG, std::string("cannot open ") + path + " for writing");
    const size_t w = std::fwrite(o.b.data(), 1, o.b.size(), fp);
    const int c = std::fclose(fp);
    if (w != o.b.size() || c != 0) return mat_fail(IMG_ERR_ARG, std::string("short write to ") + path);
    return IMG_OK;
}

int img_slice_read(const char* path, int grid[3], double* mass, double* mom, double* ener, double* mag,
                   int* has_mag) {
    if (!path || !grid) return mat_fail(IMG_ERR_ARG, "null argument");
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return mat_fail(IMG_ERR_ARG, std::string("cannot open ") + path);
    std::vector<uint8_t> buf;
    uint8_t chunk[1 << 16];
    size_t r;
    while ((r = std::fread(chunk, 1, sizeof chunk, fp)) > 0) buf.insert(buf.end(), chunk, chunk + r);
    std::fclose(fp);
    if (buf.size() < 128 || buf[126] != 'I' || buf[127] != 'M')
        return mat_fail(IMG_ERR_ARG, "not a little-endian MAT-file Level 5");
    In in{buf.data(), buf.size(), 128};
    uint32_t t;
    std::vector<uint8_t> d;
    Node var;
    std::string name;
    bool found = false;
    while (!found && next_element(in, t, d)) {   // the first variable (data.(fields{1}))
        if (t != miMATRIX && t != miCOMPRESSED) continue;
        if (!parse_value(t, d, var, name)) return mat_fail(IMG_ERR_ARG, "unreadable MAT element in " + std::string(path));
        found = true;
    }
    if (!found || var.cls != mxSTRUCT) return mat_fail(IMG_ERR_ARG, "no slice struct in " + std::string(path));
    const Node* ms = field(var, "mass");
    const Node* en = field(var, "ener");
    const Node* px[3] = {field(var, "momX"), field(var, "momY"), field(var, "momZ")};
    const Node* bx[3] = {field(var, "magX"), field(var, "magY"), field(var, "magZ")};
    if (!ms || !en || !px[0] || !px[1] || !px[2]) return mat_fail(IMG_ERR_ARG, "slice lacks mass, ener or momentum");
    std::vector<int> dims = ms->dims;
    while (dims.size() < 3) dims.push_back(1);
    if (dims.size() > 3) return mat_fail(IMG_ERR_ARG, "mass has more than 3 dimensions");
    const size_t n = ms->num.size();
    for (int k = 0; k < 3; ++k) grid[k] = dims[k];
    const bool hm = bx[0] && !bx[0]->num.empty();
    if (has_mag) *has_mag = hm ? 1 : 0;
    auto same = [&](const Node* a) { return a && a->num.size() == n; };
    if (!same(en) || !same(px[0]) || !same(px[1]) || !same(px[2]))
        return mat_fail(IMG_ERR_ARG, "slice arrays differ in size");
    if (hm && !(same(bx[0]) && same(bx[1]) && same(bx[2]))) return mat_fail(IMG_ERR_ARG, "magnet arrays differ in size");
    if (mass) std::memcpy(mass, ms->num.data(), n * 8);
    if (ener) std::memcpy(ener, en->num.data(), n * 8);
    for (int c = 0; c < 3; ++c) {
        if (mom) std::memcpy(mom + c * n, px[c]->num.data(), n * 8);
        if (mag) {
            if (hm) std::memcpy(mag + c * n, bx[c]->num.data(), n * 8);
            else std::memset(mag + c * n, 0, n * 8);
        }
    }
    return IMG_OK;
}

}  // extern "C"
