// The on-disk grid Hamiltonian (Hmt.xml / Hmt.json) that a43 exports and the Green-function
// code reads: grid, boundary conditions, spacing, the local potential on the full grid and the
// SHO atoms with their Hamiltonian and overlap matrices.
//
// Reader: the fields green_input::load_Hamiltonian takes from the XML file (src/green_input.cxx:
// 29-221) and json_reading::load_Hamiltonian from the JSON file (include/json_reading.hxx:61-229),
// with the same defaults (spacing 1, missing potential values zero, ".json" in the name selects
// JSON and falls back to XML when that fails).  Writer: the layouts of
// grid_operators::write_to_file (include/grid_operators.hxx:460-613), number formats included.
// The reference parses with RapidXML / RapidJSON; this file carries two small parsers of its own
// for exactly these documents (elements, attributes, text and comments; objects, arrays, numbers,
// strings and literals).
#include "hamiltonian_io.hpp"

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>

namespace a43g {

namespace {

inline int nsho_of(int numax) { return ((1 + numax)*(2 + numax)*(3 + numax))/6; }

// numbers separated by white space (or commas), as strtod reads them (xml_reading::read_sequence)
std::vector<double> read_numbers(char const *s) {
    std::vector<double> v;
    char *end = nullptr;
    while (*s) {
        while (*s && (std::isspace(static_cast<unsigned char>(*s)) || ',' == *s)) ++s;
        if (!*s) break;
        errno = 0;
        double const f = std::strtod(s, &end);
        if (end == s) break;
        if (ERANGE != errno) v.push_back(f);
        s = end;
    }
    return v;
}

// ------------------------------------------------------------------ XML

struct XNode {
    std::string name, text;
    std::map<std::string, std::string> attr;
    std::vector<std::unique_ptr<XNode>> kids;
    XNode const *child(char const *n) const {
        for (auto const &k : kids) if (k->name == n) return k.get();
        return nullptr;
    }
    char const *get(char const *a, char const *def = "") const {
        auto const it = attr.find(a);
        return (attr.end() == it) ? def : it->second.c_str();
    }
};

class XmlParser {
  public:
    explicit XmlParser(std::string const &s) : s_(s) {}
    std::unique_ptr<XNode> parse(std::string &err) {
        auto root = std::unique_ptr<XNode>(new XNode());
        root->name = "#document";
        if (!content(*root, err)) return nullptr;
        return root;
    }
  private:
    std::string const &s_;
    size_t p_ = 0;
    bool starts(char const *t) const { return 0 == s_.compare(p_, std::strlen(t), t); }
    void ws() { while (p_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[p_]))) ++p_; }
    bool skip_until(char const *t) {
        size_t const q = s_.find(t, p_);
        if (std::string::npos == q) return false;
        p_ = q + std::strlen(t);
        return true;
    }
    std::string name() {
        size_t const q = p_;
        while (p_ < s_.size() && (std::isalnum(static_cast<unsigned char>(s_[p_])) || std::strchr("_-.:", s_[p_]))) ++p_;
        return s_.substr(q, p_ - q);
    }
    // children and text of node until its end tag (or the end of the document)
    bool content(XNode &node, std::string &err) {
        while (p_ < s_.size()) {
            if ('<' != s_[p_]) {
                size_t const q = s_.find('<', p_);
                node.text.append(s_, p_, (std::string::npos == q ? s_.size() : q) - p_);
                p_ = (std::string::npos == q) ? s_.size() : q;
                continue;
            }
            if (starts("<!--")) { if (!skip_until("-->")) { err = "unterminated comment"; return false; } continue; }
            if (starts("<?")) { if (!skip_until("?>")) { err = "unterminated declaration"; return false; } continue; }
            if (starts("<!")) { if (!skip_until(">")) { err = "unterminated markup"; return false; } continue; }
            if (starts("</")) {
                p_ += 2;
                std::string const n = name();
                ws();
                if (p_ >= s_.size() || '>' != s_[p_]) { err = "bad end tag </" + n; return false; }
                ++p_;
                if (n != node.name) { err = "end tag </" + n + "> does not close <" + node.name + ">"; return false; }
                return true;
            }
            ++p_;                                    // '<'
            auto kid = std::unique_ptr<XNode>(new XNode());
            kid->name = name();
            if (kid->name.empty()) { err = "bad element name"; return false; }
            for (;;) {
                ws();
                if (p_ >= s_.size()) { err = "unterminated element <" + kid->name; return false; }
                if (starts("/>")) { p_ += 2; break; }
                if ('>' == s_[p_]) {
                    ++p_;
                    if (!content(*kid, err)) return false;
                    break;
                }
                std::string const a = name();
                ws();
                if (a.empty() || p_ >= s_.size() || '=' != s_[p_]) { err = "bad attribute in <" + kid->name; return false; }
                ++p_; ws();
                char const q = (p_ < s_.size()) ? s_[p_] : 0;
                if ('"' != q && '\'' != q) { err = "unquoted attribute in <" + kid->name; return false; }
                size_t const e = s_.find(q, p_ + 1);
                if (std::string::npos == e) { err = "unterminated attribute in <" + kid->name; return false; }
                kid->attr[a] = s_.substr(p_ + 1, e - p_ - 1);
                p_ = e + 1;
            }
            node.kids.push_back(std::move(kid));
        }
        if ("#document" != node.name) { err = "missing </" + node.name + ">"; return false; }
        return true;
    }
};

// ------------------------------------------------------------------ JSON

struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    double num = 0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;
    JVal const *member(char const *k) const {
        for (auto const &m : obj) if (m.first == k) return &m.second;
        return nullptr;
    }
};

class JsonParser {
  public:
    explicit JsonParser(std::string const &s) : s_(s) {}
    bool parse(JVal &v, std::string &err) {
        if (!value(v, err)) return false;
        ws();
        if (p_ != s_.size()) { err = "trailing characters after the JSON value"; return false; }
        return true;
    }
  private:
    std::string const &s_;
    size_t p_ = 0;
    void ws() { while (p_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[p_]))) ++p_; }
    bool string(std::string &out, std::string &err) {
        ++p_;                                        // '"'
        while (p_ < s_.size() && '"' != s_[p_]) {
            if ('\\' == s_[p_] && p_ + 1 < s_.size()) { out += s_[p_ + 1]; p_ += 2; continue; }
            out += s_[p_++];
        }
        if (p_ >= s_.size()) { err = "unterminated string"; return false; }
        ++p_;
        return true;
    }
    bool value(JVal &v, std::string &err) {
        ws();
        if (p_ >= s_.size()) { err = "unexpected end of the JSON text"; return false; }
        char const c = s_[p_];
        if ('{' == c) {
            v.kind = JVal::Obj; ++p_; ws();
            if (p_ < s_.size() && '}' == s_[p_]) { ++p_; return true; }
            for (;;) {
                ws();
                if (p_ >= s_.size() || '"' != s_[p_]) { err = "object key expected"; return false; }
                std::string k;
                if (!string(k, err)) return false;
                ws();
                if (p_ >= s_.size() || ':' != s_[p_]) { err = "':' expected after \"" + k + "\""; return false; }
                ++p_;
                v.obj.emplace_back(k, JVal());
                if (!value(v.obj.back().second, err)) return false;
                ws();
                if (p_ < s_.size() && ',' == s_[p_]) { ++p_; continue; }
                if (p_ < s_.size() && '}' == s_[p_]) { ++p_; return true; }
                err = "',' or '}' expected in an object"; return false;
            }
        }
        if ('[' == c) {
            v.kind = JVal::Arr; ++p_; ws();
            if (p_ < s_.size() && ']' == s_[p_]) { ++p_; return true; }
            for (;;) {
                v.arr.emplace_back();
                if (!value(v.arr.back(), err)) return false;
                ws();
                if (p_ < s_.size() && ',' == s_[p_]) { ++p_; continue; }
                if (p_ < s_.size() && ']' == s_[p_]) { ++p_; return true; }
                err = "',' or ']' expected in an array"; return false;
            }
        }
        if ('"' == c) { v.kind = JVal::Str; return string(v.str, err); }
        if (0 == s_.compare(p_, 4, "true")) { v.kind = JVal::Bool; v.num = 1; p_ += 4; return true; }
        if (0 == s_.compare(p_, 5, "false")) { v.kind = JVal::Bool; v.num = 0; p_ += 5; return true; }
        if (0 == s_.compare(p_, 4, "null")) { v.kind = JVal::Null; p_ += 4; return true; }
        char *end = nullptr;
        v.num = std::strtod(s_.c_str() + p_, &end);
        if (end == s_.c_str() + p_) { err = "bad JSON value"; return false; }
        v.kind = JVal::Num;
        p_ = size_t(end - s_.c_str());
        return true;
    }
};

std::vector<double> json_numbers(JVal const *v) {
    std::vector<double> out;
    if (!v) return out;
    if (JVal::Num == v->kind || JVal::Bool == v->kind) { out.push_back(v->num); return out; }
    if (JVal::Arr == v->kind)
        for (auto const &e : v->arr) { auto const sub = json_numbers(&e); out.insert(out.end(), sub.begin(), sub.end()); }
    return out;
}

bool read_file(char const *filename, std::string &text) {
    std::ifstream f(filename, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    text = ss.str();
    return true;
}

std::string load_xml(std::string const &text, Hamiltonian &h) {
    std::string err;
    XmlParser parser(text);
    auto const doc = parser.parse(err);
    if (!doc) return "XML: " + err;
    auto const gh = doc->child("grid_Hamiltonian");
    if (!gh) return "no <grid_Hamiltonian> element";
    h = Hamiltonian{};
    if (auto const atoms = gh->child("sho_atoms")) {
        int const number = std::atoi(atoms->get("number", "0"));
        for (auto const &atom : atoms->kids) {
            if ("atom" != atom->name) continue;
            double a8[8] = {0, 0, 0, 0, 0, -1, -1, 0};
            a8[3] = std::atof(atom->get("Z", "0"));
            a8[4] = std::atoi(atom->get("global_id", "-1"));
            if (auto const pos = atom->child("position")) {
                char const *const xyz[3] = {"x", "y", "z"};
                for (int d = 0; d < 3; ++d) a8[d] = std::atof(pos->get(xyz[d], "0"));
            }
            if (auto const prj = atom->child("projectors")) {
                a8[5] = std::atoi(prj->get("numax", "-1"));
                a8[6] = std::atof(prj->get("sigma", "-1"));
            }
            int const numax = int(a8[5]);
            if (numax < 0) return "an atom without <projectors numax>";
            int const nc = nsho_of(numax);
            std::vector<double> m(2*size_t(nc)*nc, 0.0);
            char const *const tags[2] = {"hamiltonian", "overlap"};
            for (int hs = 0; hs < 2; ++hs) {
                auto const mat = atom->child(tags[hs]);
                if (!mat) continue;                  // a missing matrix stays zero (the reference warns)
                auto const v = read_numbers(mat->text.c_str());
                if (v.size() != size_t(nc)*nc)
                    return std::string(tags[hs]) + " matrix of atom " + std::to_string(int(a8[4])) + " has " +
                           std::to_string(v.size()) + " values, expected " + std::to_string(nc*nc);
                std::copy(v.begin(), v.end(), m.begin() + size_t(hs)*nc*nc);
            }
            h.xyzZinso.insert(h.xyzZinso.end(), a8, a8 + 8);
            h.atom_mat.push_back(std::move(m));
        }
        if (int(h.atom_mat.size()) != number) return "<sho_atoms number> differs from the atoms found";
    }
    if (auto const sp = gh->child("spacing")) {
        char const *const xyz[3] = {"x", "y", "z"};
        for (int d = 0; d < 3; ++d) { char const *v = sp->get(xyz[d]); if (*v) h.hg[d] = std::atof(v); }
    }
    if (auto const bc = gh->child("boundary")) {
        char const *const xyz[3] = {"x", "y", "z"};
        for (int d = 0; d < 3; ++d) { char const *v = bc->get(xyz[d]); if (*v) h.bc[d] = std::atoi(v); }
    }
    if (auto const pot = gh->child("potential")) {
        char const *const n[3] = {"nx", "ny", "nz"};
        for (int d = 0; d < 3; ++d) { char const *v = pot->get(n[d]); if (*v) h.ng[d] = uint32_t(std::atoi(v)); }
        h.Veff = read_numbers(pot->text.c_str());
    }
    h.Veff.resize(size_t(h.ng[0])*h.ng[1]*h.ng[2], 0.0);   // missing values are zero (reference default)
    return "";
}

std::string load_json(std::string const &text, Hamiltonian &h) {
    std::string err;
    JVal doc;
    JsonParser parser(text);
    if (!parser.parse(doc, err)) return "JSON: " + err;
    if (JVal::Obj != doc.kind) return "JSON: the document is not an object";
    h = Hamiltonian{};
    auto const sp = json_numbers(doc.member("spacing"));
    for (size_t d = 0; d < 3 && d < sp.size(); ++d) h.hg[d] = sp[d];
    auto const bc = json_numbers(doc.member("boundary"));
    for (size_t d = 0; d < 3 && d < bc.size(); ++d) h.bc[d] = int(bc[d]);
    if (auto const pot = doc.member("potential")) {
        auto const g = json_numbers(pot->member("grid"));
        for (size_t d = 0; d < 3 && d < g.size(); ++d) h.ng[d] = uint32_t(g[d]);
        h.Veff = json_numbers(pot->member("values"));
    }
    h.Veff.resize(size_t(h.ng[0])*h.ng[1]*h.ng[2], 0.0);
    if (auto const sa = doc.member("sho_atoms")) {
        auto const num = json_numbers(sa->member("number"));
        int const number = num.empty() ? 0 : int(num[0]);
        if (auto const atoms = sa->member("atoms")) {
            for (auto const &atom : atoms->arr) {
                double a8[8] = {0, 0, 0, 0, 0, -1, 1, 0};
                auto const id = json_numbers(atom.member("atom_id"));
                if (!id.empty()) a8[4] = id[0];
                if (auto const prj = atom.member("projectors")) {
                    auto const nu = json_numbers(prj->member("numax"));
                    auto const sg = json_numbers(prj->member("sigma"));
                    if (!nu.empty()) a8[5] = nu[0];
                    if (!sg.empty()) a8[6] = sg[0];
                }
                auto const pos = json_numbers(atom.member("position"));
                if (3 == pos.size()) for (int d = 0; d < 3; ++d) a8[d] = pos[d];
                int const numax = int(a8[5]);
                if (numax < 0) return "an atom without projectors.numax";
                int const nc = nsho_of(numax);
                std::vector<double> m(2*size_t(nc)*nc, 0.0);
                char const *const tags[2] = {"hamiltonian", "overlap"};
                for (int hs = 0; hs < 2; ++hs) {
                    auto const v = json_numbers(atom.member(tags[hs]));
                    if (v.empty()) continue;
                    if (v.size() != size_t(nc)*nc)
                        return std::string(tags[hs]) + " matrix with " + std::to_string(v.size()) + " values, expected " +
                               std::to_string(nc*nc);
                    std::copy(v.begin(), v.end(), m.begin() + size_t(hs)*nc*nc);
                }
                h.xyzZinso.insert(h.xyzZinso.end(), a8, a8 + 8);
                h.atom_mat.push_back(std::move(m));
            }
        }
        if (int(h.atom_mat.size()) != number) return "sho_atoms.number differs from the atoms found";
    }
    return "";
}

} // namespace

std::string Hamiltonian::load(char const *filename) {
    std::string text;
    if (!filename || !read_file(filename, text)) return std::string("cannot read \"") + (filename ? filename : "") + "\"";
    if (std::strstr(filename, ".json")) {
        auto const e = load_json(text, *this);
        if (e.empty()) return "";
        auto const x = load_xml(text, *this);   // as the reference: try XML when JSON fails
        return x.empty() ? "" : e;
    }
    return load_xml(text, *this);
}

std::string Hamiltonian::save(char const *filename, bool json, double const *spectrum) const {
    FILE *f = std::fopen(filename, "w");
    if (!f) return std::string("cannot write \"") + filename + "\"";
    size_t const natoms = atom_mat.size(), nall = size_t(ng[0])*ng[1]*ng[2];
    if (!json) {
        std::fprintf(f, "<?xml version=\"%.1f\"?>\n", 1.0);
        std::fprintf(f, "<grid_Hamiltonian version=\"%.1f\">\n", 0.);
        std::fprintf(f, "  <!-- Units: Hartree and Bohr radii. -->\n");
        if (spectrum) std::fprintf(f, "  <spectrum min=\"%.6f\" max=\"%.6f\" Fermi=\"%.6f\" unit=\"Hartree\"/>\n",
                                   spectrum[0], spectrum[1], spectrum[2]);
        std::fprintf(f, "  <sho_atoms number=\"%ld\">\n", long(natoms));
        for (size_t ia = 0; ia < natoms; ++ia) {
            double const *a = &xyzZinso[8*ia];
            std::fprintf(f, "    <atom global_id=\"%i\" Z=\"%d\">\n", int(a[4]), int(std::lround(a[3])));
            std::fprintf(f, "      <position x=\"%.12f\" y=\"%.12f\" z=\"%.12f\" unit=\"Bohr\"/>\n", a[0], a[1], a[2]);
            int const numax = int(a[5]), nc = nsho_of(numax);
            std::fprintf(f, "      <projectors type=\"sho\" numax=\"%d\" sigma=\"%.12f\" unit=\"Bohr\"/>\n", numax, a[6]);
            for (int hs = 0; hs < 2; ++hs) {
                double const *m = atom_mat[ia].data() + size_t(hs)*nc*nc;
                char const *tag = hs ? "overlap" : "hamiltonian";
                std::fprintf(f, "      <%s unit=\"%s\">\n", tag, hs ? "1" : "Hartree");
                for (int i = 0; i < nc; ++i) {
                    std::fprintf(f, "        ");
                    for (int j = 0; j < nc; ++j) {
                        if (hs && 0 == m[i*nc + j]) std::fprintf(f, " 0");   // exact zeros abbreviated
                        else std::fprintf(f, " %.15e", m[i*nc + j]);
                    }
                    std::fprintf(f, "\n");
                }
                std::fprintf(f, "      </%s>\n", tag);
            }
            std::fprintf(f, "    </atom>\n");
        }
        std::fprintf(f, "  </sho_atoms>\n");
        std::fprintf(f, "  <spacing x=\"%.17f\" y=\"%.17f\" z=\"%.17f\" unit=\"Bohr\"/>\n", hg[0], hg[1], hg[2]);
        std::fprintf(f, "  <boundary x=\"%d\" y=\"%d\" z=\"%d\"/>\n", bc[0], bc[1], bc[2]);
        double vmin = 0, vmax = 0, vsum = 0;
        for (size_t i = 0; i < nall; ++i) {
            vmin = i ? std::min(vmin, Veff[i]) : Veff[i]; vmax = i ? std::max(vmax, Veff[i]) : Veff[i]; vsum += Veff[i];
        }
        std::fprintf(f, "  <potential nx=\"%d\" ny=\"%d\" nz=\"%d\" minimum=\"%g\" maximum=\"%g\" average=\"%g\" unit=\"Hartree\">",
                     int(ng[0]), int(ng[1]), int(ng[2]), vmin, vmax, nall ? vsum/nall : 0.0);
        for (size_t i = 0; i < nall; ++i) {
            if (0 == (i & 3)) std::fprintf(f, "\n    ");
            std::fprintf(f, " %.15f", Veff[i]);
        }
        std::fprintf(f, "\n  </potential>\n");
        std::fprintf(f, "</grid_Hamiltonian>\n");
    } else {
        std::fprintf(f, "{\n");
        std::fprintf(f, "  \"comment\": \"grid_Hamiltonian in units of Hartree and Bohr radii\"\n");
        if (spectrum) std::fprintf(f, "  ,\"spectrum\": {\"min\": %.6f, \"max\": %.6f, \"Fermi\": %.6f}\n",
                                   spectrum[0], spectrum[1], spectrum[2]);
        std::fprintf(f, " ,\"sho_atoms\":\n  {\n");
        std::fprintf(f, "    \"number\": %ld\n", long(natoms));
        std::fprintf(f, "   ,\"atoms\": [\n");
        for (size_t ia = 0; ia < natoms; ++ia) {
            double const *a = &xyzZinso[8*ia];
            std::fprintf(f, "     %c{\"atom_id\": %i\n", ia ? ',' : ' ', int(a[4]));
            std::fprintf(f, "      ,\"Z\": %d\n", int(std::lround(a[3])));
            std::fprintf(f, "      ,\"position\": [%.12f, %.12f, %.12f]\n", a[0], a[1], a[2]);
            int const numax = int(a[5]), nc = nsho_of(numax);
            std::fprintf(f, "      ,\"projectors\": {\"type\": \"sho\", \"numax\": %d, \"sigma\": %.12f}\n", numax, a[6]);
            for (int hs = 0; hs < 2; ++hs) {
                double const *m = atom_mat[ia].data() + size_t(hs)*nc*nc;
                std::fprintf(f, "      ,\"%s\":\n", hs ? "overlap" : "hamiltonian");
                for (int i = 0; i < nc; ++i) {
                    std::fprintf(f, "        %c", i ? ',' : '[');
                    for (int j = 0; j < nc; ++j) {
                        if (0 == (j & 3)) std::fprintf(f, "\n          ");
                        if (0 == m[i*nc + j]) std::fprintf(f, "%c0", j ? ',' : '[');
                        else std::fprintf(f, "%c%.15e", j ? ',' : '[', m[i*nc + j]);
                    }
                    std::fprintf(f, "]\n");
                }
                std::fprintf(f, "        ]\n");
            }
            std::fprintf(f, "      }\n");
        }
        std::fprintf(f, "    ]\n");
        std::fprintf(f, "  }\n");
        std::fprintf(f, " ,\"spacing\": [%.17f, %.17f, %.17f]\n", hg[0], hg[1], hg[2]);
        std::fprintf(f, " ,\"boundary\": [%d, %d, %d]\n", bc[0], bc[1], bc[2]);
        std::fprintf(f, " ,\"potential\": {\n");
        std::fprintf(f, "    \"grid\": [%d, %d, %d]\n", int(ng[0]), int(ng[1]), int(ng[2]));
        std::fprintf(f, "   ,\"values\":");
        for (size_t i = 0; i < nall; ++i) {
            if (0 == (i & 3)) std::fprintf(f, "\n    ");
            std::fprintf(f, "%c%.15f", i ? ',' : '[', Veff[i]);
        }
        std::fprintf(f, "]\n");
        std::fprintf(f, "  }\n");
        std::fprintf(f, "}\n");
    }
    bool const ok = 0 == std::ferror(f);
    std::fclose(f);
    return ok ? "" : std::string("error writing \"") + filename + "\"";
}

} // namespace a43g
