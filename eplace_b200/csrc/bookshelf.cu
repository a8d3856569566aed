// bookshelf.cu -- native Bookshelf reader and full-precision writers for
// the engine's array netlist.  Host code only; no CUDA call.
//
// The reader restates what Parser/parser.cpp:44-819 takes from a design:
//   .aux   "RowBasedPlacement : a.nodes a.nets a.wts a.pl a.scl" (files by
//          extension; .wts is not read, as the reference ignores net weights)
//   .nodes "name w h [terminal | terminal_NI]" after a header line; the
//          NumNodes / NumTerminals lines and '#' comments are skipped
//          (parser.cpp:271-440: terminals and terminal_NI are fixed pads,
//          the latter flagged not-in-image)
//   .nets  "NetDegree : d [name]" followed by d pin lines
//          "owner dir [: dx dy]" (offset from the owner's centre, 0 when absent)
//   .pl    "name llx lly [: orient] [/FIXED...]" lower-left corners; '(', ')',
//          ',', ':' and '=' are separators; a name that .nodes does not
//          define is skipped (the reference exits, parser.cpp:799)
//   .scl   CoreRow blocks: Coordinate (row bottom), Height, Sitewidth (kept
//          for later rows), "SubrowOrigin : x Numsites : n" (row end
//          x + n * Sitewidth, parser.cpp:211-230)
// The arrays it fills are those of ep_netlist: movable nodes first, in file
// order, then the terminals in file order; node centres are the .pl corner
// plus half the size in float, as Module::setLocation_2D
// (PlaceCommon/objects.cpp:518-527).
// The Python reader eplace_b200/bookshelf.py states the same rules and the
// tests compare the two array for array.
#include <cctype>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <string_view>
#include <system_error>
#include <unordered_map>
#include <vector>

#include "eplace_gpu.h"

namespace {

struct BookshelfDesign {
    std::vector<std::string> names;  // output order: movable nodes, then terminals
    std::vector<float> node_w, node_h, node_cx, node_cy;
    std::vector<float> term_llx, term_lly, term_w, term_h;
    std::vector<uint8_t> term_ni;
    std::vector<int32_t> net_start, pin_owner;
    std::vector<float> pin_dx, pin_dy;
    std::vector<float> row_llx, row_lly, row_urx, row_h;
    std::vector<float> row_site_w;  // not part of ep_netlist; kept for the writer
};

struct ParseError {
    std::string msg;
};

bool read_file(const std::string &path, std::string &out) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (n < 0) {
        std::fclose(f);
        return false;
    }
    out.resize((size_t)n);
    const bool ok = std::fread(&out[0], 1, (size_t)n, f) == (size_t)n;
    std::fclose(f);
    return ok;
}

// Lines of a buffer; get() returns false at the end.
struct Lines {
    const char *p, *end;
    explicit Lines(const std::string &s) : p(s.data()), end(s.data() + s.size()) {}
    bool get(std::string_view &line) {
        if (p >= end) return false;
        const char *q = static_cast<const char *>(std::memchr(p, '\n', (size_t)(end - p)));
        if (!q) q = end;
        line = std::string_view(p, (size_t)(q - p));
        p = q < end ? q + 1 : end;
        return true;
    }
};

// Character classes of a tokenizer: 0 part of a token, 1 separator
// (whitespace and the extra characters given), 2 a token of its own.
struct CharClass {
    uint8_t c[256];
    CharClass(const char *drop, const char *own) {
        for (int i = 0; i < 256; i++) c[i] = std::isspace(i) ? 1 : 0;
        for (; *drop; drop++) c[(unsigned char)*drop] = 1;
        for (; *own; own++) c[(unsigned char)*own] = 2;
    }
};
const CharClass kPlain("", ""), kNets("", ":"), kPl("(),:=\r", "");

// Tokens of a line under the given character classes.
void tokens(std::string_view line, std::vector<std::string_view> &out, const CharClass &cls = kPlain) {
    out.clear();
    size_t i = 0;
    const size_t n = line.size();
    const uint8_t *c = cls.c;
    while (i < n) {
        while (i < n && c[(unsigned char)line[i]] == 1) i++;
        if (i >= n) break;
        if (c[(unsigned char)line[i]] == 2) {
            out.push_back(line.substr(i, 1));
            i++;
            continue;
        }
        size_t j = i;
        while (j < n && c[(unsigned char)line[j]] == 0) j++;
        out.push_back(line.substr(i, j - i));
        i = j;
    }
}

// A decimal number filling the whole token, correctly rounded to double
// (as strtod and Python's float); a leading '+' is accepted.
double number(std::string_view t, const char *what) {
    const char *b = t.data(), *e = t.data() + t.size();
    if (b < e && *b == '+') b++;
    double v = 0;
    const auto r = std::from_chars(b, e, v);
    if (b == e || r.ec != std::errc() || r.ptr != e)
        throw ParseError{"bad number '" + std::string(t) + "' for " + what};
    return v;
}

// Node name -> index of its last .nodes line: open addressing over the
// 64-bit hash (FNV-1a), the name compared only when the hashes agree.
struct NameIndex {
    std::vector<uint64_t> key;  // hash | 1; 0 = empty slot
    std::vector<int32_t> val;
    const std::vector<std::string_view> *names = nullptr;
    size_t mask = 0;

    static uint64_t hash(std::string_view s) {
        uint64_t h = 1469598103934665603ull;
        for (unsigned char c : s) h = (h ^ c) * 1099511628211ull;
        h ^= h >> 29;  // spread the low bits the slot index uses
        return h | 1;
    }
    void build(const std::vector<std::string_view> &n) {
        names = &n;
        size_t cap = 16;
        while (cap < 2 * n.size()) cap <<= 1;
        key.assign(cap, 0);
        val.assign(cap, -1);
        mask = cap - 1;
        for (size_t i = 0; i < n.size(); i++) {
            const uint64_t h = hash(n[i]);
            size_t s = h & mask;
            while (key[s] && !(key[s] == h && (*names)[val[s]] == n[i])) s = (s + 1) & mask;
            key[s] = h;
            val[s] = (int32_t)i;  // a repeated name refers to its last line
        }
    }
    int32_t find(std::string_view name) const {
        const uint64_t h = hash(name);
        for (size_t s = h & mask; key[s]; s = (s + 1) & mask)
            if (key[s] == h && (*names)[val[s]] == name) return val[s];
        return -1;
    }
};

bool starts_with(std::string_view s, const char *p) { return s.substr(0, std::strlen(p)) == p; }

struct Parsed {
    std::vector<std::string_view> names;  // file order
    std::vector<float> w, h, llx, lly;
    std::vector<int> kind;  // 0 node, 1 terminal, 2 terminal_NI
    NameIndex index;
};

void parse_nodes(const std::string &buf, Parsed &d) {
    Lines ls(buf);
    std::string_view line;
    std::vector<std::string_view> t;
    ls.get(line);  // header
    while (ls.get(line)) {
        tokens(line, t);
        if (t.empty() || t[0][0] == '#' || t[0] == "NumNodes" || t[0] == "NumTerminals") continue;
        if (t.size() < 3) throw ParseError{"short line in .nodes: '" + std::string(line) + "'"};
        d.names.push_back(t[0]);
        d.w.push_back((float)number(t[1], "node width"));
        d.h.push_back((float)number(t[2], "node height"));
        int k = 0;
        if (t.size() > 3 && starts_with(t[3], "terminal")) k = t[3] == "terminal_NI" ? 2 : 1;
        d.kind.push_back(k);
    }
    d.index.build(d.names);
}

void parse_nets(const std::string &buf, const Parsed &d, const std::vector<int32_t> &remap,
                BookshelfDesign &out) {
    Lines ls(buf);
    std::string_view line;
    std::vector<std::string_view> t;
    ls.get(line);  // header
    out.net_start.assign(1, 0);
    while (ls.get(line)) {
        tokens(line, t, kNets);
        if (t.empty() || t[0][0] == '#' || t[0] == "NumNets" || t[0] == "NumPins") continue;
        if (t[0] != "NetDegree" || t.size() < 3)
            throw ParseError{"unsupported line in .nets: '" + std::string(line) + "'"};
        const long deg = std::strtol(std::string(t[2]).c_str(), nullptr, 10);
        if (deg < 0) throw ParseError{"negative net degree"};
        for (long k = 0; k < deg; k++) {
            if (!ls.get(line)) throw ParseError{"a net ends before its NetDegree pins"};
            tokens(line, t, kNets);
            if (t.empty()) throw ParseError{"empty pin line in .nets"};
            const int32_t owner = d.index.find(t[0]);
            if (owner < 0) throw ParseError{"pin of unknown node '" + std::string(t[0]) + "'"};
            out.pin_owner.push_back(remap[owner]);
            size_t c = 0;
            while (c < t.size() && t[c] != ":") c++;
            const size_t r = c + 1;  // tokens after ':'
            out.pin_dx.push_back(c < t.size() && r < t.size() ? (float)number(t[r], "pin x offset") : 0.f);
            out.pin_dy.push_back(c < t.size() && r + 1 < t.size() ? (float)number(t[r + 1], "pin y offset") : 0.f);
        }
        out.net_start.push_back((int32_t)out.pin_owner.size());
    }
}

void parse_pl(const std::string &buf, Parsed &d) {
    Lines ls(buf);
    std::string_view line;
    std::vector<std::string_view> t;
    d.llx.assign(d.names.size(), 0.f);
    d.lly.assign(d.names.size(), 0.f);
    ls.get(line);  // header
    while (ls.get(line)) {
        tokens(line, t, kPl);
        if (t.size() < 3 || t[0][0] == '#') continue;
        const int32_t i = d.index.find(t[0]);
        if (i < 0) continue;
        d.llx[i] = (float)number(t[1], "placement x");
        d.lly[i] = (float)number(t[2], "placement y");
    }
}

void parse_scl(const std::string &buf, BookshelfDesign &out) {
    struct Row {
        double bottom = 0, height = 0, site = 1, origin = 0, sites = 0;
    };
    std::vector<Row> rows;
    double site = 1.0;
    Lines ls(buf);
    std::string_view line;
    std::vector<std::string_view> t;
    auto cur = [&]() -> Row & {
        if (rows.empty()) throw ParseError{"row attribute before the first CoreRow in .scl"};
        return rows.back();
    };
    while (ls.get(line)) {
        tokens(line, t);
        if (t.empty()) continue;
        if (t[0] == "CoreRow") {
            rows.push_back(Row{});
            rows.back().site = site;
        } else if (t[0] == "Coordinate" && t.size() > 2) {
            cur().bottom = number(t[2], "row coordinate");
        } else if (t[0] == "Height" && t.size() > 2) {
            cur().height = number(t[2], "row height");
        } else if (t[0] == "Sitewidth" && t.size() > 2) {
            site = number(t[2], "site width");
            cur().site = site;
        } else if (t.size() >= 6 && (t[3] == "Numsites" || t[3] == "NumSites")) {
            cur().origin = number(t[2], "subrow origin");
            cur().sites = number(t[5], "number of sites");
        }
    }
    for (const Row &r : rows) {
        out.row_llx.push_back((float)r.origin);
        out.row_lly.push_back((float)r.bottom);
        out.row_urx.push_back((float)(r.sites * r.site + r.origin));
        out.row_h.push_back((float)r.height);
        out.row_site_w.push_back((float)r.site);
    }
}

void fail(char *errbuf, int32_t errlen, const std::string &msg) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, (size_t)errlen, "%s", msg.c_str());
}

template <typename T>
const T *data_or_null(const std::vector<T> &v) {
    return v.empty() ? nullptr : v.data();
}

// Buffered text output: numbers with std::to_chars(general, 9), which
// prints what printf("%.9g") prints, written to the file in large blocks.
class Out {
  public:
    explicit Out(const std::string &path) : f_(std::fopen(path.c_str(), "w")) { buf_.reserve(1 << 20); }
    ~Out() { close(); }
    Out &s(const char *t) {
        buf_.append(t);
        return spill();
    }
    Out &s(const std::string &t) {
        buf_.append(t);
        return spill();
    }
    Out &g(double v) {  // %.9g
        char tmp[40];
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, v, std::chars_format::general, 9);
        buf_.append(tmp, (size_t)(r.ptr - tmp));
        return spill();
    }
    Out &d(long long v) {
        char tmp[24];
        const auto r = std::to_chars(tmp, tmp + sizeof tmp, v);
        buf_.append(tmp, (size_t)(r.ptr - tmp));
        return spill();
    }
    // true when the file was opened and everything reached it
    bool close() {
        if (!f_) return false;
        flush();
        const bool ok = ok_ && std::fclose(f_) == 0;
        f_ = nullptr;
        return ok;
    }

  private:
    Out &spill() {
        if (buf_.size() >= (1 << 20)) flush();
        return *this;
    }
    void flush() {
        if (f_ && !buf_.empty()) ok_ = ok_ && std::fwrite(buf_.data(), 1, buf_.size(), f_) == buf_.size();
        buf_.clear();
    }
    FILE *f_;
    std::string buf_;
    bool ok_ = true;
};

// The .pl file: movable nodes at lower-left = centre - size/2 (float), then
// the terminals with /FIXED or /FIXED_NI; %.9g, so a float round-trips.
template <typename NameOf>
ep_status write_pl(const std::string &path, int32_t nn, int32_t nt, const float *w, const float *h, const float *cx,
                   const float *cy, const float *tllx, const float *tlly, const uint8_t *tni, NameOf name_of) {
    Out o(path);
    o.s("UCLA pl 1.0\n\n");
    for (int32_t i = 0; i < nn; i++)
        o.s(name_of(i)).s(" ").g(cx[i] - 0.5f * w[i]).s(" ").g(cy[i] - 0.5f * h[i]).s(" : N\n");
    for (int32_t k = 0; k < nt; k++)
        o.s(name_of(nn + k)).s(" ").g(tllx[k]).s(" ").g(tlly[k]).s(tni && tni[k] ? " : N /FIXED_NI\n" : " : N /FIXED\n");
    return o.close() ? EP_OK : EP_ERR_ARG;
}

}  // namespace

extern "C" {

ep_status ep_bookshelf_read(const char *aux_path, ep_netlist *nl, void **handle, char *errbuf, int32_t errlen) {
    if (!aux_path || !nl || !handle) return EP_ERR_ARG;
    *handle = nullptr;
    BookshelfDesign *out = new (std::nothrow) BookshelfDesign;
    if (!out) return EP_ERR_NOMEM;
    try {
        std::string aux;
        if (!read_file(aux_path, aux)) throw ParseError{std::string("cannot read ") + aux_path};
        std::string dir(aux_path);
        const size_t slash = dir.find_last_of('/');
        dir = slash == std::string::npos ? std::string() : dir.substr(0, slash + 1);
        std::vector<std::string_view> t;
        Lines ls(aux);
        std::string_view first;
        ls.get(first);
        tokens(first, t);
        std::unordered_map<std::string, std::string> files;  // extension -> path
        for (size_t k = 2; k < t.size(); k++) {
            const std::string name(t[k]);
            const size_t dot = name.find_last_of('.');
            if (dot != std::string::npos) files[name.substr(dot)] = dir + name;
        }
        std::string nodes, nets, pl, scl;
        const std::pair<const char *, std::string *> need[] = {
            {".nodes", &nodes}, {".nets", &nets}, {".pl", &pl}, {".scl", &scl}};
        for (auto &f : need)
            if (!files.count(f.first)) throw ParseError{std::string("the .aux names no ") + f.first + " file"};
        for (auto &f : need)
            if (!read_file(files[f.first], *f.second)) throw ParseError{"cannot read " + files[f.first]};
        Parsed d;
        parse_nodes(nodes, d);
        const int32_t n = (int32_t)d.names.size();
        std::vector<int32_t> remap(n);
        int32_t nn = 0, nt = 0;
        for (int32_t i = 0; i < n; i++)
            if (d.kind[i] == 0) remap[i] = nn++;
        for (int32_t i = 0; i < n; i++)
            if (d.kind[i] != 0) remap[i] = nn + nt++;
        parse_nets(nets, d, remap, *out);
        parse_pl(pl, d);
        parse_scl(scl, *out);
        out->names.resize(n);
        out->node_w.resize(nn);
        out->node_h.resize(nn);
        out->node_cx.resize(nn);
        out->node_cy.resize(nn);
        out->term_llx.resize(nt);
        out->term_lly.resize(nt);
        out->term_w.resize(nt);
        out->term_h.resize(nt);
        out->term_ni.resize(nt);
        for (int32_t i = 0; i < n; i++) {
            const int32_t r = remap[i];
            out->names[r] = std::string(d.names[i]);
            if (d.kind[i] == 0) {
                out->node_w[r] = d.w[i];
                out->node_h[r] = d.h[i];
                out->node_cx[r] = d.llx[i] + 0.5f * d.w[i];
                out->node_cy[r] = d.lly[i] + 0.5f * d.h[i];
            } else {
                const int32_t k = r - nn;
                out->term_llx[k] = d.llx[i];
                out->term_lly[k] = d.lly[i];
                out->term_w[k] = d.w[i];
                out->term_h[k] = d.h[i];
                out->term_ni[k] = d.kind[i] == 2;
            }
        }
        *nl = ep_netlist{};
        nl->num_nodes = nn;
        nl->num_terminals = nt;
        nl->num_nets = (int32_t)out->net_start.size() - 1;
        nl->num_rows = (int32_t)out->row_llx.size();
        nl->node_w = data_or_null(out->node_w);
        nl->node_h = data_or_null(out->node_h);
        nl->node_cx = data_or_null(out->node_cx);
        nl->node_cy = data_or_null(out->node_cy);
        nl->term_llx = data_or_null(out->term_llx);
        nl->term_lly = data_or_null(out->term_lly);
        nl->term_w = data_or_null(out->term_w);
        nl->term_h = data_or_null(out->term_h);
        nl->term_is_ni = data_or_null(out->term_ni);
        nl->net_start = out->net_start.data();
        nl->pin_owner = data_or_null(out->pin_owner);
        nl->pin_dx = data_or_null(out->pin_dx);
        nl->pin_dy = data_or_null(out->pin_dy);
        nl->row_llx = data_or_null(out->row_llx);
        nl->row_lly = data_or_null(out->row_lly);
        nl->row_urx = data_or_null(out->row_urx);
        nl->row_h = data_or_null(out->row_h);
        nl->common_row_height = 0.f;
    } catch (const ParseError &e) {
        fail(errbuf, errlen, e.msg);
        delete out;
        return EP_ERR_ARG;
    } catch (const std::bad_alloc &) {
        fail(errbuf, errlen, "out of host memory");
        delete out;
        return EP_ERR_NOMEM;
    }
    *handle = out;
    return EP_OK;
}

ep_status ep_bookshelf_write_pl(const void *handle, const char *path, const float *node_cx, const float *node_cy) try {
    const BookshelfDesign *d = static_cast<const BookshelfDesign *>(handle);
    if (!d || !path || (!d->node_w.empty() && (!node_cx || !node_cy))) return EP_ERR_ARG;
    const int32_t nn = (int32_t)d->node_w.size(), nt = (int32_t)d->term_w.size();
    return write_pl(path, nn, nt, d->node_w.data(), d->node_h.data(), node_cx, node_cy, d->term_llx.data(),
                    d->term_lly.data(), d->term_ni.data(), [&](int32_t i) -> const std::string & { return d->names[i]; });
} catch (const std::bad_alloc &) {
    return EP_ERR_NOMEM;
}

ep_status ep_bookshelf_write(const char *dir, const char *name, const ep_netlist *nl, const void *design) try {
    if (!dir || !name || !nl || nl->num_nodes < 0 || nl->num_terminals < 0 || nl->num_nets < 0 || nl->num_rows < 0)
        return EP_ERR_ARG;
    const BookshelfDesign *d = static_cast<const BookshelfDesign *>(design);
    const int32_t nn = nl->num_nodes, nt = nl->num_terminals, nnet = nl->num_nets, nr = nl->num_rows;
    if (d && ((int32_t)d->node_w.size() != nn || (int32_t)d->term_w.size() != nt)) return EP_ERR_ARG;
    const int32_t np = nnet > 0 ? nl->net_start[nnet] : 0;
    std::string tmp;
    auto node_name = [&](int32_t i) -> const std::string & {
        if (d) return d->names[i];
        tmp = (i < nn ? "o" : "t") + std::to_string(i < nn ? i : i - nn);
        return tmp;
    };
    const std::string base = std::string(dir) + "/" + name, nm(name);
    bool ok;
    {
        Out o(base + ".aux");
        o.s("RowBasedPlacement : ").s(nm + ".nodes ").s(nm + ".nets ").s(nm + ".wts ").s(nm + ".pl ");
        o.s(nm + ".scl\n");
        ok = o.close();
    }
    if (ok) {
        Out o(base + ".nodes");
        o.s("UCLA nodes 1.0\nNumNodes : ").d(nn + nt).s("\nNumTerminals : ").d(nt).s("\n");
        for (int32_t i = 0; i < nn; i++) o.s(node_name(i)).s(" ").g(nl->node_w[i]).s(" ").g(nl->node_h[i]).s("\n");
        for (int32_t k = 0; k < nt; k++)
            o.s(node_name(nn + k)).s(" ").g(nl->term_w[k]).s(" ").g(nl->term_h[k])
                .s(nl->term_is_ni && nl->term_is_ni[k] ? " terminal_NI\n" : " terminal\n");
        ok = o.close();
    }
    if (ok) {
        Out o(base + ".nets");
        o.s("UCLA nets 1.0\nNumNets : ").d(nnet).s("\nNumPins : ").d(np).s("\n");
        for (int32_t n = 0; n < nnet; n++) {
            o.s("NetDegree : ").d(nl->net_start[n + 1] - nl->net_start[n]).s(" n").d(n).s("\n");
            for (int32_t p = nl->net_start[n]; p < nl->net_start[n + 1]; p++)
                o.s(node_name(nl->pin_owner[p])).s(" B : ").g(nl->pin_dx[p]).s(" ").g(nl->pin_dy[p]).s("\n");
        }
        ok = o.close();
    }
    if (ok) {
        Out o(base + ".wts");
        o.s("UCLA wts 1.0\n");
        ok = o.close();
    }
    if (ok)
        ok = write_pl(base + ".pl", nn, nt, nl->node_w, nl->node_h, nl->node_cx, nl->node_cy, nl->term_llx,
                      nl->term_lly, nl->term_is_ni, node_name) == EP_OK;
    if (ok) {
        Out o(base + ".scl");
        o.s("UCLA scl 1.0\nNumRows : ").d(nr).s("\n");
        for (int32_t r = 0; r < nr; r++) {
            const float site = d && (int32_t)d->row_site_w.size() == nr ? d->row_site_w[r] : 1.f;
            const float sites = (nl->row_urx[r] - nl->row_llx[r]) / site;
            o.s("CoreRow Horizontal\n Coordinate : ").g(nl->row_lly[r]).s("\n Height : ").g(nl->row_h[r]);
            o.s("\n Sitewidth : ").g(site).s("\n Sitespacing : ").g(site);
            o.s("\n Siteorient : N\n Sitesymmetry : Y\n SubrowOrigin : ").g(nl->row_llx[r]).s(" Numsites : ");
            o.g(sites).s("\nEnd\n");
        }
        ok = o.close();
    }
    return ok ? EP_OK : EP_ERR_ARG;
} catch (const std::bad_alloc &) {
    return EP_ERR_NOMEM;
}

ep_status ep_bookshelf_row_site_widths(const void *handle, float *out, int32_t count) {
    const BookshelfDesign *d = static_cast<const BookshelfDesign *>(handle);
    if (!d || count < 0 || (size_t)count != d->row_site_w.size() || (count > 0 && !out)) return EP_ERR_ARG;
    for (int32_t r = 0; r < count; r++) out[r] = d->row_site_w[r];
    return EP_OK;
}

void ep_bookshelf_close(void *handle) { delete static_cast<BookshelfDesign *>(handle); }

}  // extern "C"
