// scheme_xml.cpp -- the reference's scheme files, read without Mini-XML.
//
// Scheme::load_from_file (common-lib/scheme.cpp:272-857) reads an XML file
// whose element texts hold the values: one <general> (name, result_file,
// optional log_file), <surface> elements (class, type, shape, params, size,
// center, distance, angles, optional comment; grating_type, order, const,
// n1, n2 for gratings; n1, n2 for lenses; AUX surfaces only distance and
// angles) and one <beam> (type, shape, profile, range_distr, params, center,
// range, optional nlambda).  A value is the text of the first element of that
// name below the node (mxmlFindPath), with spaces and tabs trimmed
// (scheme.cpp:30-44,151-174); numbers are read with strtod until it stops
// (scheme.cpp:178-210), "strict" fields must be numbers only, and a strict
// field that is not a number is a file name (n1, n2 tables; the range file).
//
// This reader builds the same values with a small XML parser of its own:
// elements, text, comments, processing instructions and the five predefined
// entities.  Surfaces are taken in document order; Mini-XML's index
// (mxmlIndexNew/mxmlIndexFind, scheme.cpp:399-402) is what the reference
// iterates, and whether it yields document order is a property of that
// library this code cannot check.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/rtb.h"

extern "C" RTB_API int rtb_spline_init(size_t n, const double* x, const double* y, double* y2);

namespace {

// ---- a minimal XML tree ---------------------------------------------------------

struct Node {
    std::string name;
    std::string text;  // text before the first child element (the "opaque" value)
    bool has_text = false;
    std::vector<std::unique_ptr<Node>> kids;
};

struct Parser {
    const std::string& s;
    size_t i = 0;
    bool ok = true;
    explicit Parser(const std::string& src) : s(src) {}

    bool starts(const char* t) const { return s.compare(i, std::strlen(t), t) == 0; }

    void skip_misc() {  // comments, declarations, processing instructions, whitespace
        for (;;) {
            while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
            if (starts("<!--")) {
                size_t e = s.find("-->", i + 4);
                if (e == std::string::npos) { ok = false; return; }
                i = e + 3;
            } else if (starts("<?")) {
                size_t e = s.find("?>", i + 2);
                if (e == std::string::npos) { ok = false; return; }
                i = e + 2;
            } else if (starts("<!")) {
                size_t e = s.find('>', i + 2);
                if (e == std::string::npos) { ok = false; return; }
                i = e + 1;
            } else {
                return;
            }
        }
    }

    static void decode(std::string& t) {
        static const struct { const char* e; char c; } ents[] = {
            {"&lt;", '<'}, {"&gt;", '>'}, {"&amp;", '&'}, {"&quot;", '"'}, {"&apos;", '\''}};
        std::string o;
        o.reserve(t.size());
        for (size_t k = 0; k < t.size();) {
            bool hit = false;
            if (t[k] == '&')
                for (const auto& e : ents) {
                    size_t n = std::strlen(e.e);
                    if (t.compare(k, n, e.e) == 0) {
                        o += e.c;
                        k += n;
                        hit = true;
                        break;
                    }
                }
            if (!hit) o += t[k++];
        }
        t.swap(o);
    }

    std::unique_ptr<Node> element() {
        if (i >= s.size() || s[i] != '<') { ok = false; return nullptr; }
        ++i;
        auto n = std::make_unique<Node>();
        while (i < s.size() && !std::isspace((unsigned char)s[i]) && s[i] != '>' && s[i] != '/') n->name += s[i++];
        // attributes are not used by the scheme format: skip them
        while (i < s.size() && s[i] != '>' && !(s[i] == '/' && i + 1 < s.size() && s[i + 1] == '>')) {
            if (s[i] == '"' || s[i] == '\'') {
                size_t e = s.find(s[i], i + 1);
                if (e == std::string::npos) { ok = false; return nullptr; }
                i = e + 1;
            } else {
                ++i;
            }
        }
        if (i >= s.size()) { ok = false; return nullptr; }
        if (s[i] == '/') {  // <name/>
            i += 2;
            return n;
        }
        ++i;  // '>'
        bool first = true;
        for (;;) {
            size_t t0 = i;
            while (i < s.size() && s[i] != '<') ++i;
            if (i >= s.size()) { ok = false; return nullptr; }
            if (first && i > t0) {
                n->text = s.substr(t0, i - t0);
                decode(n->text);
                n->has_text = true;
            }
            if (starts("<!--")) {
                size_t e = s.find("-->", i + 4);
                if (e == std::string::npos) { ok = false; return nullptr; }
                i = e + 3;
                continue;
            }
            if (starts("</")) {
                size_t e = s.find('>', i);
                if (e == std::string::npos) { ok = false; return nullptr; }
                std::string closing = s.substr(i + 2, e - i - 2);
                while (!closing.empty() && std::isspace((unsigned char)closing.back())) closing.pop_back();
                if (closing != n->name) { ok = false; return nullptr; }
                i = e + 1;
                return n;
            }
            first = false;
            auto k = element();
            if (!ok) return nullptr;
            n->kids.push_back(std::move(k));
        }
    }
};

// First element called `name` below `n`, depth first in document order.
const Node* find(const Node* n, const std::string& name) {
    for (const auto& k : n->kids) {
        if (k->name == name) return k.get();
        if (const Node* d = find(k.get(), name)) return d;
    }
    return nullptr;
}

void find_all(const Node* n, const std::string& name, std::vector<const Node*>& out) {
    for (const auto& k : n->kids) {
        if (k->name == name) out.push_back(k.get());
        find_all(k.get(), name, out);
    }
}

// ---- values (scheme.cpp:30-48,128-210) ------------------------------------------

enum SchemeError {  // Scheme::SchemeError (scheme.h:25-27)
    FileOpenFailure, ParseFailure, NoClassAttr, BadAttrValue, NanAttrValue, MemAllocFailure,
    NoSchemeDesc, NoBeamDesc, NoSurfaceDesc, NoRange, NoRangeFile, BadRange,
    EmptyScheme, BadStartIndex, FileSaveFailure
};

struct Fail {
    int code;
};

std::string value(const Node* at, const char* name, bool upper = true) {
    const Node* e = find(at, name);
    if (!e) throw Fail{ParseFailure};
    if (!e->has_text) throw Fail{BadAttrValue};
    std::string v = e->text;
    const char* ws = " \t";
    size_t b = v.find_first_not_of(ws);
    if (b == std::string::npos) throw Fail{BadAttrValue};
    v = v.substr(b, v.find_last_not_of(ws) - b + 1);
    if (upper)
        for (auto& c : v) c = (char)std::toupper((unsigned char)c);
    return v;
}

std::vector<double> numbers(const Node* at, const char* name, bool strict = false) {
    std::string v = value(at, name);
    const char* p = v.c_str();
    std::vector<double> out;
    for (;;) {
        char* e = nullptr;
        double x = std::strtod(p, &e);
        if (e == p) break;
        out.push_back(x);
        p = e;
    }
    if (strict && *p != '\0') throw Fail{NanAttrValue};
    if (out.empty()) throw Fail{BadAttrValue};
    return out;
}

// AsciiFile::ReadLine (common-lib/ascii_file.cpp): '#' comment lines and
// blank lines skipped; a line that does not start with `need` numbers is
// invalid.  The reference reads lines with getline and stops at end of file
// before looking at the line it was reading, so a last line without a
// newline is not read; that is kept.
int read_rows(const std::string& path, size_t need, std::vector<std::vector<double>>& rows) {
    std::ifstream f(path);
    if (!f) return -1;
    std::string line;
    while (std::getline(f, line)) {
        if (f.eof()) break;  // the reference drops an unterminated last line
        size_t k = 0;
        while (k < line.size() && line[k] == ' ') ++k;
        if (k == line.size()) continue;
        if (line[k] == '#') continue;
        const char* p = line.c_str() + k;
        std::vector<double> v;
        for (size_t j = 0; j < need; ++j) {
            char* e = nullptr;
            double x = std::strtod(p, &e);
            if (e == p) return -2;
            v.push_back(x);
            p = e;
        }
        rows.push_back(v);
    }
    return 0;
}

}  // namespace

struct rtb_scheme {
    std::string name, result_file, log_file;
    std::vector<std::string> comments;
    std::vector<rtb_surface> surfaces;
    std::vector<std::vector<double>> tables;  // x | y | y2 of every file table, and single values
    rtb_scheme_beam beam{};
    std::vector<double> ranges;  // rows of row_len numbers
    size_t row_len = 0;
    std::vector<rtb_qe_surface> qe;  // ComputeQE's surfaces
    int qe_error = -1;               // SchemeError ComputeQE meets on them, -1 none
};

namespace {

// A refractive index: a number, or a table file (TabulatedFunction::Load,
// tabulated_function.cpp:58-118: at least 4 rows, x strictly increasing,
// natural-spline second derivatives).
void index_table(rtb_scheme& sc, const Node* at, const char* name, const std::string& dir, rtb_table& t) {
    std::string file;
    try {
        std::vector<double> v = numbers(at, name, true);
        sc.tables.push_back({v[0]});
        t.n = 1;
        t.y = sc.tables.back().data();
        t.x = t.y2 = nullptr;
        return;
    } catch (Fail&) {
        file = value(at, name, false);
    }
    std::vector<std::vector<double>> rows;
    int r = read_rows(file, 2, rows);
    if (r == -1 && !dir.empty() && file[0] != '/') r = read_rows(dir + "/" + file, 2, rows);
    if (r != 0 || rows.size() < 4) throw Fail{BadAttrValue};
    const size_t n = rows.size();
    std::vector<double> tab(3 * n);
    for (size_t k = 0; k < n; ++k) {
        tab[k] = rows[k][0];
        tab[n + k] = rows[k][1];
        if (k && !(tab[k] > tab[k - 1])) throw Fail{BadAttrValue};
    }
    if (rtb_spline_init(n, tab.data(), tab.data() + n, tab.data() + 2 * n) != RTB_OK) throw Fail{BadAttrValue};
    sc.tables.push_back(std::move(tab));
    const double* b = sc.tables.back().data();
    t.n = n;
    t.x = b;
    t.y = b + n;
    t.y2 = b + 2 * n;
}

// The surfaces of Scheme::ComputeQE (scheme.cpp:1140-1209): non-AUX surfaces
// of type MIRROR, LENS, GRATING or DETECTOR with their qe_curve, gratings with
// alpha, gamma, blaze_angle, const, order and rule_params, read in that order.
// qe_curve is a number, or else a table file (a missing attribute is an
// error, scheme.cpp:1194-1201); a number must be > 0 (TabulatedFunction::Set,
// tabulated_function.cpp:121-137).  rule_params: none gives 0 1, one value v
// gives 0 v, both clamped to [0, 1] and start < stop required
// (Grating::SetRuleParams, surface.cpp:595-611).
void load_qe(const std::vector<const Node*>& surf, const std::string& dir, rtb_scheme& sc) {
    for (const Node* s : surf) {
        if (value(s, "class") == "AUX") continue;
        const std::string type = value(s, "type");
        rtb_qe_surface q;
        std::memset(&q, 0, sizeof(q));
        if (type == "MIRROR") q.type = RTB_MIRROR;
        else if (type == "LENS") q.type = RTB_LENS;
        else if (type == "GRATING") q.type = RTB_GRATING;
        else if (type == "DETECTOR") q.type = RTB_DETECTOR;
        else continue;
        if (q.type == RTB_GRATING) {
            q.alpha_deg = numbers(s, "alpha")[0];
            q.gamma_deg = numbers(s, "gamma")[0];
            q.blaze_deg = numbers(s, "blaze_angle")[0];
            q.gr_const = numbers(s, "const")[0];
            q.order = (int64_t)(long)numbers(s, "order")[0];
            std::vector<double> rp;
            try {
                rp = numbers(s, "rule_params", true);
                if (rp.size() == 1) rp.insert(rp.begin(), 0.0);
            } catch (Fail&) {
                rp = {0.0, 1.0};
            }
            q.rule_start = rp[0];
            q.rule_stop = rp[1];
            const double a = std::min(std::max(rp[0], 0.0), 1.0), b = std::min(std::max(rp[1], 0.0), 1.0);
            if (a >= b) throw Fail{BadAttrValue};
        }
        index_table(sc, s, "qe_curve", dir, q.qe);
        if (q.qe.n == 1 && !(q.qe.y[0] > 0.0)) throw Fail{BadAttrValue};
        sc.qe.push_back(q);
    }
    if (sc.qe.empty()) throw Fail{NoSurfaceDesc};
}

void load(const std::string& path, rtb_scheme& sc) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw Fail{FileOpenFailure};
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string src = ss.str();
    Parser p(src);
    auto root = std::make_unique<Node>();
    p.skip_misc();
    while (p.ok && p.i < src.size()) {
        auto e = p.element();
        if (!p.ok) break;
        root->kids.push_back(std::move(e));
        p.skip_misc();
    }
    if (!p.ok) throw Fail{ParseFailure};
    const std::string dir = path.find('/') == std::string::npos ? "" : path.substr(0, path.rfind('/'));

    const Node* gen = find(root.get(), "general");
    if (!gen) throw Fail{NoSchemeDesc};
    sc.name = value(gen, "name", false);
    sc.result_file = value(gen, "result_file", false);
    try {
        sc.log_file = value(gen, "log_file", false);
    } catch (Fail&) {
        sc.log_file.clear();
    }

    std::vector<const Node*> surf;
    find_all(root.get(), "surface", surf);
    if (surf.empty()) throw Fail{NoSurfaceDesc};
    if (surf.size() > RTB_MAX_SURFACES) throw Fail{BadAttrValue};
    sc.tables.reserve(3 * surf.size() + 1);  // pointers into it stay valid
    int n_gratings = 0;
    for (const Node* s : surf) {
        rtb_surface o;
        std::memset(&o, 0, sizeof(o));
        o.n1.n = o.n2.n = 0;
        const std::string cls = value(s, "class");
        std::string type = "AUX", shape = "CIRC";
        std::vector<double> params, size, center;
        if (cls != "AUX") {
            type = value(s, "type");
            shape = value(s, "shape");
            params = numbers(s, "params");
            size = numbers(s, "size");
            center = numbers(s, "center");
        }
        std::vector<double> dist = numbers(s, "distance"), ang = numbers(s, "angles");
        if (cls == "PLANE") o.cls = RTB_PLANE;
        else if (cls == "CONIC") o.cls = RTB_CONIC;
        else if (cls == "TORIC") o.cls = RTB_TORIC;
        else if (cls == "AUX") o.cls = RTB_AUX_CLASS;
        else throw Fail{BadAttrValue};
        if (type == "MIRROR") o.type = RTB_MIRROR;
        else if (type == "LENS") o.type = RTB_LENS;
        else if (type == "GRATING") o.type = RTB_GRATING;
        else if (type == "STOP") o.type = RTB_STOP;
        else if (type == "SHADE") o.type = RTB_SHADE;
        else if (type == "DETECTOR") o.type = RTB_DETECTOR;
        else if (type == "AUX") o.type = RTB_AUX_TYPE;
        else throw Fail{BadAttrValue};
        if (shape.compare(0, 4, "CIRC") == 0) o.shape = RTB_CIRCLE;
        else if (shape.compare(0, 4, "RECT") == 0) o.shape = RTB_RECTANGLE;
        else throw Fail{BadAttrValue};
        std::string comment;
        try {
            comment = value(s, "comment", false);
        } catch (Fail&) {
        }
        sc.comments.push_back(comment);
        if (o.type == RTB_GRATING) {
            // missing or empty: reflective; any other word is an error (the
            // reference throws Grating::BadType past its handler, scheme.cpp:512-523)
            o.grating_type = RTB_REFLECTIVE;
            std::string g;
            try {
                g = value(s, "grating_type");
            } catch (Fail&) {
                g = "REFLECTIVE";
            }
            if (g == "TRANSPARENT") o.grating_type = RTB_TRANSPARENT;
            else if (g != "REFLECTIVE") throw Fail{BadAttrValue};
            o.order = (int64_t)numbers(s, "order")[0];
            o.gr_const = numbers(s, "const")[0];
            ++n_gratings;
        }
        if (o.type == RTB_GRATING || o.type == RTB_LENS) {
            index_table(sc, s, "n1", dir, o.n1);
            index_table(sc, s, "n2", dir, o.n2);
        }
        // Surface::SetDistance / SetAngles / SetParams / SetGeometry: the first
        // three distances and angles, up to RTB_MAX_PARAMS parameters
        for (size_t k = 0; k < 3; ++k) {
            o.distance[k] = k < dist.size() ? dist[k] : 0.0;
            o.angles_deg[k] = k < ang.size() ? ang[k] : 0.0;
        }
        if (params.size() > RTB_MAX_PARAMS) throw Fail{BadAttrValue};
        for (size_t k = 0; k < params.size(); ++k) o.params[k] = params[k];
        for (size_t k = 0; k < 2; ++k) {
            o.size[k] = k < size.size() ? size[k] : 0.0;
            o.center[k] = k < center.size() ? center[k] : 0.0;
        }
        sc.surfaces.push_back(o);
    }

    const Node* beam = find(root.get(), "beam");
    if (!beam) throw Fail{NoBeamDesc};
    const std::string btype = value(beam, "type"), bshape = value(beam, "shape"), bprof = value(beam, "profile"),
                      bdist = value(beam, "range_distr");
    std::vector<double> bpars = numbers(beam, "params"), bcen = numbers(beam, "center");
    // range: "w1 w2 [orders]" or a file of such rows (scheme.cpp:213-256)
    try {
        std::vector<double> v = numbers(beam, "range", true);
        if (v.size() < 2 || v[0] >= v[1] || v[1] <= 0.0) throw Fail{BadRange};
        sc.row_len = v.size();
        sc.ranges = v;
    } catch (Fail& e) {
        if (e.code != NanAttrValue) throw;
        const std::string file = value(beam, "range", false);
        std::vector<std::vector<double>> rows;
        int r = read_rows(file, 2 + n_gratings, rows);
        if (r == -1 && !dir.empty() && file[0] != '/') r = read_rows(dir + "/" + file, 2 + n_gratings, rows);
        if (r == -1) throw Fail{NoRangeFile};
        if (r != 0) throw Fail{BadRange};
        for (const auto& v : rows)
            if (v[0] >= v[1] || v[0] <= 0.0 || v[1] <= 0.0) throw Fail{BadRange};
        if (rows.empty()) throw Fail{BadRange};
        sc.row_len = 2 + n_gratings;
        for (const auto& v : rows) sc.ranges.insert(sc.ranges.end(), v.begin(), v.end());
    }
    rtb_scheme_beam& b = sc.beam;
    if (btype == "PARALLEL") b.type = RTB_BEAM_PARALLEL;
    else if (btype == "CONIC") b.type = RTB_BEAM_CONIC;
    else if (btype == "GAUSS") b.type = RTB_BEAM_GAUSS;
    else throw Fail{BadAttrValue};
    if (bshape.compare(0, 4, "CIRC") == 0) b.shape = RTB_CIRCLE;
    else if (bshape.compare(0, 4, "RECT") == 0) b.shape = RTB_RECTANGLE;
    else throw Fail{BadAttrValue};
    if (bprof == "RANDOM") b.profile = RTB_PROFILE_RANDOM;
    else if (bprof == "CONCENTRIC") b.profile = RTB_PROFILE_CONCENTRIC;
    else throw Fail{BadAttrValue};
    if (bdist == "RANDOM") b.range_distr = RTB_RANGE_RANDOM;
    else if (bdist == "UNIFORM") b.range_distr = RTB_RANGE_UNIFORM;
    else if (bdist == "MONOCHROMATIC") b.range_distr = RTB_RANGE_MONOCHROMATIC;
    else throw Fail{BadAttrValue};
    b.n_params = (int32_t)(bpars.size() < 6 ? bpars.size() : 6);
    for (int k = 0; k < b.n_params; ++k) b.params[k] = bpars[k];
    for (size_t k = 0; k < 3; ++k) b.center[k] = k < bcen.size() ? bcen[k] : 0.0;
    b.n_lambda = 0;
    if (b.range_distr != RTB_RANGE_MONOCHROMATIC) {
        try {
            b.n_lambda = (uint64_t)numbers(beam, "nlambda", true)[0];
        } catch (Fail&) {
            b.n_lambda = 0;
        }
    }
    // ComputeQE's own attributes: a scheme that traces may lack them
    try {
        load_qe(surf, dir, sc);
    } catch (Fail& e) {
        sc.qe.clear();
        sc.qe_error = e.code;
    }
}

}  // namespace

extern "C" {

RTB_API int rtb_scheme_load(const char* path, rtb_scheme** out, int* scheme_error) {
    if (scheme_error) *scheme_error = -1;
    if (!path || !out) return RTB_BAD_VALUE;
    *out = nullptr;
    rtb_scheme* sc = new (std::nothrow) rtb_scheme();
    if (!sc) return RTB_BAD_ALLOC;
    try {
        load(path, *sc);
    } catch (Fail& e) {
        if (scheme_error) *scheme_error = e.code;
        delete sc;
        return RTB_BAD_VALUE;
    } catch (std::bad_alloc&) {
        if (scheme_error) *scheme_error = MemAllocFailure;
        delete sc;
        return RTB_BAD_ALLOC;
    }
    *out = sc;
    return RTB_OK;
}

RTB_API int rtb_scheme_surfaces(const rtb_scheme* sc, const rtb_surface** surfaces, size_t* n) {
    if (!sc || !surfaces || !n) return RTB_BAD_VALUE;
    *surfaces = sc->surfaces.data();
    *n = sc->surfaces.size();
    return RTB_OK;
}

RTB_API const char* rtb_scheme_text(const rtb_scheme* sc, int which) {
    if (!sc) return nullptr;
    if (which == RTB_SCHEME_NAME) return sc->name.c_str();
    if (which == RTB_SCHEME_RESULT_FILE) return sc->result_file.c_str();
    if (which == RTB_SCHEME_LOG_FILE) return sc->log_file.c_str();
    const int k = which - RTB_SCHEME_COMMENT;
    if (k >= 0 && k < (int)sc->comments.size()) return sc->comments[k].c_str();
    return nullptr;
}

RTB_API int rtb_scheme_get_beam(const rtb_scheme* sc, rtb_scheme_beam* beam) {
    if (!sc || !beam) return RTB_BAD_VALUE;
    *beam = sc->beam;
    return RTB_OK;
}

RTB_API int rtb_scheme_ranges(const rtb_scheme* sc, const double** rows, size_t* n_rows, size_t* row_len) {
    if (!sc || !rows || !n_rows || !row_len) return RTB_BAD_VALUE;
    *rows = sc->ranges.data();
    *row_len = sc->row_len;
    *n_rows = sc->row_len ? sc->ranges.size() / sc->row_len : 0;
    return RTB_OK;
}

RTB_API void rtb_scheme_free(rtb_scheme* sc) { delete sc; }

RTB_API int rtb_scheme_qe_surfaces(const rtb_scheme* sc, const rtb_qe_surface** surfaces, size_t* n,
                                   int* scheme_error) {
    if (scheme_error) *scheme_error = -1;
    if (!sc || !surfaces || !n) return RTB_BAD_VALUE;
    *surfaces = nullptr;
    *n = 0;
    if (sc->qe_error >= 0) {
        if (scheme_error) *scheme_error = sc->qe_error;
        return RTB_BAD_VALUE;
    }
    *surfaces = sc->qe.data();
    *n = sc->qe.size();
    return RTB_OK;
}

RTB_API int rtb_save_qe(const char* path, size_t n_rows, size_t n_lambda, const double* lambda, const double* qe) {
    if (!path || (n_rows && n_lambda && (!lambda || !qe))) return RTB_BAD_VALUE;
    FILE* f = std::fopen(path, "wb");
    if (!f) return RTB_BAD_VALUE;
    bool ok = true;
    for (size_t r = 0; r < n_rows && ok; ++r) {
        ok = std::fwrite(&n_lambda, sizeof(size_t), 1, f) == 1 &&
             std::fwrite(lambda + r * n_lambda, sizeof(double), n_lambda, f) == n_lambda &&
             std::fwrite(qe + r * n_lambda, sizeof(double), n_lambda, f) == n_lambda;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? RTB_OK : RTB_BAD_VALUE;
}

}  // extern "C"
