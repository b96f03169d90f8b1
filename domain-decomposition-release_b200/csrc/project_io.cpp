// project_io.cpp -- see project_io.hpp.  A small reader for the flat JSON
// object of argfile.json (strings, numbers, booleans; // and /* */
// comments) written for this library: the reference links jsoncpp for the
// same twelve keys.
#include "project_io.hpp"

#include <cctype>
#include <cstdint>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace jv {

namespace {

struct JsonVal {
    enum Kind { kStr, kNum, kBool, kNull } kind = kNull;
    std::string s;
    double n = 0;
    bool b = false;
};

std::string strip_comments(const std::string &t) {
    std::string o;
    o.reserve(t.size());
    bool in_str = false;
    for (size_t i = 0; i < t.size();) {
        char c = t[i];
        if (in_str) {
            o += c;
            if (c == '\\' && i + 1 < t.size()) {
                o += t[i + 1];
                i += 2;
                continue;
            }
            if (c == '"') in_str = false;
            i++;
        } else if (c == '"') {
            in_str = true;
            o += c;
            i++;
        } else if (t.compare(i, 2, "//") == 0) {
            size_t j = t.find('\n', i);
            i = (j == std::string::npos) ? t.size() : j;
        } else if (t.compare(i, 2, "/*") == 0) {
            size_t j = t.find("*/", i + 2);
            i = (j == std::string::npos) ? t.size() : j + 2;
        } else {
            o += c;
            i++;
        }
    }
    return o;
}

struct Parser {
    const std::string &t;
    size_t i = 0;
    std::string err;
    explicit Parser(const std::string &s) : t(s) {}
    void ws() {
        while (i < t.size() && std::isspace((unsigned char)t[i])) i++;
    }
    bool str(std::string *out) {
        if (i >= t.size() || t[i] != '"') return false;
        i++;
        std::string o;
        while (i < t.size() && t[i] != '"') {
            if (t[i] == '\\' && i + 1 < t.size()) {
                char e = t[i + 1];
                o += (e == 'n') ? '\n' : (e == 't') ? '\t' : e;
                i += 2;
            } else {
                o += t[i++];
            }
        }
        if (i >= t.size()) return false;
        i++;
        *out = o;
        return true;
    }
    bool value(JsonVal *v) {
        ws();
        if (i >= t.size()) return false;
        if (t[i] == '"') {
            v->kind = JsonVal::kStr;
            return str(&v->s);
        }
        if (t.compare(i, 4, "true") == 0) {
            v->kind = JsonVal::kBool;
            v->b = true;
            i += 4;
            return true;
        }
        if (t.compare(i, 5, "false") == 0) {
            v->kind = JsonVal::kBool;
            v->b = false;
            i += 5;
            return true;
        }
        if (t.compare(i, 4, "null") == 0) {
            v->kind = JsonVal::kNull;
            i += 4;
            return true;
        }
        const char *b = t.c_str() + i;
        char *e = nullptr;
        errno = 0;
        double d = std::strtod(b, &e);
        if (e == b || errno == ERANGE) return false;
        v->kind = JsonVal::kNum;
        v->n = d;
        i += (size_t)(e - b);
        return true;
    }
    bool object(std::map<std::string, JsonVal> *m) {
        ws();
        if (i >= t.size() || t[i] != '{') return false;
        i++;
        ws();
        if (i < t.size() && t[i] == '}') {
            i++;
            return true;
        }
        for (;;) {
            ws();
            std::string k;
            if (!str(&k)) return false;
            ws();
            if (i >= t.size() || t[i] != ':') return false;
            i++;
            JsonVal v;
            if (!value(&v)) return false;
            (*m)[k] = v;
            ws();
            if (i < t.size() && t[i] == ',') {
                i++;
                continue;
            }
            if (i < t.size() && t[i] == '}') {
                i++;
                return true;
            }
            return false;
        }
    }
};

}  // namespace

std::string read_argfile(const std::string &proj_path_in, ArgFile *a) {
    std::string proj = proj_path_in;
    if (!proj.empty() && proj.back() != '/') proj += '/';
    std::ifstream f(proj + "argfile.json");
    if (!f.is_open()) return "argfile open error: " + proj + "argfile.json";
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = strip_comments(ss.str());
    Parser p(text);
    std::map<std::string, JsonVal> m;
    if (!p.object(&m)) return "argfile.json: malformed JSON near offset " + std::to_string(p.i);
    auto gs = [&](const char *k) -> std::string {
        auto it = m.find(k);
        return (it != m.end() && it->second.kind == JsonVal::kStr) ? it->second.s : std::string();
    };
    auto gi = [&](const char *k, int d) -> int {
        auto it = m.find(k);
        return (it != m.end() && it->second.kind == JsonVal::kNum) ? (int)it->second.n : d;
    };
    auto gf = [&](const char *k) -> float {
        auto it = m.find(k);
        return (it != m.end() && it->second.kind == JsonVal::kNum) ? (float)it->second.n : 0.f;
    };
    // path values are prefixed with proj_path (fdtd3d_base_1_interface.hpp:60-62,75)
    a->proj_path = proj;
    a->model_path = proj + gs("model_path");
    a->shot_path = proj + gs("shot_path");
    a->recv_path = proj + gs("rece_path");
    a->output_path = proj + gs("output_path");
    a->x_divide_num = gi("x_divide_num", 1);
    a->y_divide_num = gi("y_divide_num", 1);
    a->z_divide_num = gi("z_divide_num", 1);
    a->slots_per_node = gi("slots_per_node", 1);
    a->pml_num = gi("pml_num", 0);
    a->t_snap = gi("t_snap", -1);
    a->fm = gf("fm");
    a->T = gf("T");
    a->dt = gf("dt");
    auto io = m.find("is_output");
    a->is_output = io != m.end() && io->second.kind == JsonVal::kBool && io->second.b;
    a->rec_width = gi("rec_width", 0);
    a->precision = gs("precision");
    if (!gs("vp_path").empty()) {
        a->vp_path = proj + gs("vp_path");
        a->vs_path = proj + gs("vs_path");
        a->rho_path = proj + gs("rho_path");
        a->n_rows = gi("n_rows", 0);
        a->n_cols = gi("n_cols", 0);
        a->n_slices = gi("n_slices", 0);
        a->d_rows = gf("d_rows");
        a->d_cols = gf("d_cols");
        a->d_slices = gf("d_slices");
        if (a->n_rows <= 0 || a->n_cols <= 0 || a->n_slices <= 0 || !(a->d_rows > 0) || !(a->d_cols > 0) ||
            !(a->d_slices > 0))
            return "argfile.json: a raw model (vp_path) needs n_rows, n_cols, n_slices > 0 and d_rows, d_cols, "
                   "d_slices > 0";
    }
    auto sf = m.find("save_fld");
    a->save_fld = sf != m.end() && sf->second.kind == JsonVal::kBool && sf->second.b;
    return "";
}

std::string read_raw(const std::string &path, float *out, size_t n) {
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) return "raw file open error: " + path;
    std::fseek(fp, 0, SEEK_END);
    const long long bytes = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (bytes != (long long)(n * sizeof(float))) {
        std::fclose(fp);
        return path + ": " + std::to_string(bytes) + " bytes, the frame needs " + std::to_string(n * sizeof(float));
    }
    const size_t r = std::fread(out, sizeof(float), n, fp);
    std::fclose(fp);
    return r == n ? "" : path + ": short read";
}

std::string read_raw_model(const ArgFile &a, GmsModel *m) {
    m->nx = a.n_rows;
    m->ny = a.n_cols;
    m->nz = a.n_slices;
    m->dx = a.d_rows; m->dy = a.d_cols; m->dz = a.d_slices;
    m->lx = m->ly = m->lz = 0.f;
    const size_t n = (size_t)m->nx * m->ny * m->nz;
    m->params.assign(3, std::vector<float>(n));
    const std::string *paths[3] = {&a.vp_path, &a.vs_path, &a.rho_path};
    for (int q = 0; q < 3; q++) {
        std::string e = read_raw(*paths[q], m->params[q].data(), n);
        if (!e.empty()) return e;
    }
    return "";
}

std::string read_points(const std::string &path, std::vector<float> *xyz) {
    std::ifstream f(path);
    if (!f.is_open()) return "geometry file open error: " + path;
    long long n = -1;
    if (!(f >> n) || n < 0) return path + ": missing point count";
    xyz->resize((size_t)n * 3);
    for (long long i = 0; i < 3 * n; i++)
        if (!(f >> (*xyz)[(size_t)i])) return path + ": expected " + std::to_string(n) + " points";
    return "";
}

#pragma pack(push, 1)
struct GmsHeader {  // GmsFileHeader (jarvis_device_gms_bones.hpp:6-29), natural alignment spelled out
    int16_t format;
    char name[64];
    int16_t year;
    char mon, day, hour, minutes, seconds, type;
    int16_t para_num;
    float l_rows, l_cols, l_slices;
    uint32_t n_rows, n_cols, n_slices;
    float d_rows, d_cols, d_slices;
    char reserved[128];
};
#pragma pack(pop)
static_assert(sizeof(GmsHeader) == 240, "GMS header is 240 bytes");

std::string read_gms(const std::string &path, GmsModel *m) {
    FILE *fp = std::fopen(path.c_str(), "rb");
    if (!fp) return "GMS open error: " + path;
    GmsHeader h;
    if (std::fread(&h, 240, 1, fp) != 1) {
        std::fclose(fp);
        return path + ": short GMS header";
    }
    if (h.para_num < 3 || h.n_rows == 0 || h.n_cols == 0 || h.n_slices == 0) {
        std::fclose(fp);
        return path + ": GMS model needs vp, vs, rho on a non-empty grid";
    }
    m->nx = (int)h.n_rows;
    m->ny = (int)h.n_cols;
    m->nz = (int)h.n_slices;
    m->dx = h.d_rows; m->dy = h.d_cols; m->dz = h.d_slices;
    m->lx = h.l_rows; m->ly = h.l_cols; m->lz = h.l_slices;
    const size_t n = (size_t)m->nx * m->ny * m->nz;
    std::vector<float> buf(n);
    m->params.clear();
    for (int p = 0; p < h.para_num; p++) {
        char name[64];
        if (std::fread(name, 64, 1, fp) != 1 || std::fread(buf.data(), sizeof(float), n, fp) != n) {
            std::fclose(fp);
            return path + ": truncated GMS data";
        }
        // data[i*nz + j*nx*nz + k] -> x-fastest field (jarvis_device_gms_meat.hpp:41-52)
        std::vector<float> f(n);
        for (int k = 0; k < m->nz; k++)
            for (int j = 0; j < m->ny; j++)
                for (int i = 0; i < m->nx; i++)
                    f[(size_t)i + (size_t)m->nx * ((size_t)j + (size_t)m->ny * k)] =
                        buf[(size_t)i * m->nz + (size_t)j * m->nx * m->nz + k];
        m->params.push_back(std::move(f));
    }
    std::fclose(fp);
    return "";
}

std::string size_info(int nx, int ny, int nz, float lx, float ly, float lz) {
    return "_" + std::to_string(nx) + "_" + std::to_string(ny) + "_" + std::to_string(nz) + "_" +
           std::to_string(lx) + "_" + std::to_string(ly) + "_" + std::to_string(lz);
}

std::string write_traces(const std::string &path_noext, const float *tr, int nrec, int nt) {
    std::string path = path_noext + ".txt";
    FILE *fp = std::fopen(path.c_str(), "wt");
    if (!fp) return "cannot create " + path;
    for (int r = 0; r < nrec; r++) {
        for (int t = 0; t < nt; t++) std::fprintf(fp, "%10.6e\t", tr[(size_t)r * nt + t]);
        std::fprintf(fp, "\n");
    }
    std::fclose(fp);
    return "";
}

std::string write_raw(const std::string &path, const float *a, size_t n) {
    FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) return "cannot create " + path;
    size_t w = std::fwrite(a, sizeof(float), n, fp);
    std::fclose(fp);
    return w == n ? "" : "short write " + path;
}

}  // namespace jv
