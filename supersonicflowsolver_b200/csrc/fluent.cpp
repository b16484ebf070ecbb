// Fluent ASCII mesh reader.
//
// Accepts the sections PSST's reader understands (psstAnsysDirector::build_step,
// psstAnsysGridReader.cpp:1138-1306): 2 dimension, 10 vertices, 12 cells,
// 13 faces, 39/45 zone names, 58/59 cell/face trees of adapted meshes. Header fields are parsed the way private_parse_number does
// (:1319-1374) and, like the reference, a header line that does not end with
// '(' consumes the following line before the data are read. Unlike the
// reference, CR characters are treated as whitespace, so CRLF files load.
//
// The whole file is read into memory once and scanned with a hand-written
// hex tokenizer: face sections of large meshes are tens of millions of hex
// integers.
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "host.hpp"

namespace psst {

int64_t RawMesh::zone_slot(int64_t id) {
    for (size_t i = 0; i < zones.size(); ++i)
        if (zones[i].id == id) return (int64_t)i;
    Zone z;
    z.id = id;
    zones.push_back(z);
    return (int64_t)zones.size() - 1;
}

namespace {

struct Cursor {
    const char *p, *end;
    bool eof() const { return p >= end; }
    static bool ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }
    void skip_ws() {
        while (p < end && ws(*p)) ++p;
    }
    // std::getline without the newline, CR stripped at the end
    void line(const char *&b, const char *&e) {
        b = p;
        while (p < end && *p != '\n') ++p;
        e = p;
        if (p < end) ++p;
        while (e > b && e[-1] == '\r') --e;
    }
    bool hex(int64_t &v) {
        skip_ws();
        int64_t x = 0;
        const char *s = p;
        for (; p < end; ++p) {
            char c = *p;
            int d;
            if (c >= '0' && c <= '9')
                d = c - '0';
            else if (c >= 'a' && c <= 'f')
                d = c - 'a' + 10;
            else if (c >= 'A' && c <= 'F')
                d = c - 'A' + 10;
            else
                break;
            x = x * 16 + d;
        }
        if (p == s) return false;
        v = x;
        return true;
    }
    bool dbl(double &v) {
        skip_ws();
        if (p >= end) return false;
        char *e;
        v = std::strtod(p, &e);  // correctly rounded, as operator>>(double&)
        if (e == p) return false;
        p = e;
        return true;
    }
};

struct Header {  // a section header line and the parse position in it
    const char *b, *e;
    const char *pos;
    int64_t number(int base) {
        char buf[64];
        int k = 0;
        bool empty = true;
        int64_t dest = 0;
        while (pos < e) {
            char c = *pos;
            bool digit = (c >= '0' && c <= '9') ||
                         (base == 16 && ((c >= 'a' && c <= 'f') || (c >= 'A' && c <= 'F')));
            if (digit) {
                if (k < 63) buf[k++] = c;
                empty = false;
            } else if (c == ' ' || c == '(' || c == ')') {
                if (!empty) {
                    buf[k] = 0;
                    dest = std::strtoll(buf, nullptr, base);
                    break;
                }
            } else {
                break;
            }
            ++pos;
        }
        return dest;
    }
    std::string name() {
        std::string out;
        bool empty = true;
        while (pos < e) {
            char c = *pos;
            if (c != ' ' && c != '(' && c != ')') {
                out.push_back(c);
                empty = false;
            } else if (!empty) {
                break;
            }
            ++pos;
        }
        return out;
    }
    bool ends_with_paren() const {
        for (const char *q = e; q > b;) {
            --q;
            if (*q == ' ' || *q == '\t') continue;
            return *q == '(';
        }
        return false;
    }
};

}  // namespace

RawMesh read_fluent(const std::string &path) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) raise(PSST_ERR_IO, "Error: Could not open \"" + path + "\" file!");
    std::fseek(f, 0, SEEK_END);
    long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)n + 1);
    size_t got = std::fread(buf.data(), 1, (size_t)n, f);
    std::fclose(f);
    buf[got] = 0;

    RawMesh m;
    Cursor c{buf.data(), buf.data() + got};
    auto fmt = [&](const std::string &what) { raise(PSST_ERR_FORMAT, path + ": " + what); };
    while (!c.eof()) {
        Header h;
        c.line(h.b, h.e);
        h.pos = h.b;
        int64_t op = h.number(10);
        if (op == 2) {
            m.dim = (int)h.number(16);
        } else if (op == 10) {
            int64_t zid = h.number(16), first = h.number(16), last = h.number(16);
            h.number(16);
            h.number(16);
            if (zid == 0) continue;
            if (!h.ends_with_paren()) {
                const char *b, *e;
                c.line(b, e);
            }
            if (m.dim != 2 && m.dim != 3) fmt("vertex section before a valid dimension section");
            int64_t cnt = last - first + 1;
            size_t base = m.verts.size();
            m.verts.resize(base + (size_t)cnt * m.dim);
            for (int64_t i = 0; i < cnt * m.dim; ++i)
                if (!c.dbl(m.verts[base + i])) fmt("truncated vertex section");
        } else if (op == 12) {
            int64_t zid = h.number(16), first = h.number(16), last = h.number(16);
            int64_t bc = h.number(16), type = h.number(16);
            if (zid == 0) continue;
            if (!h.ends_with_paren()) {
                const char *b, *e;
                c.line(b, e);
            }
            Zone &z = m.zones[m.zone_slot(zid)];
            z.first = first;
            z.last = last;
            z.bc = bc;
            z.size = last - first + 1;
            for (int64_t i = 0; i < z.size; ++i) {
                int64_t t = type;
                if (type == 0 && !c.hex(t)) fmt("truncated cell section");
                m.cell_zone.push_back(zid);
                m.cell_type.push_back(t);
            }
        } else if (op == 13) {
            int64_t zid = h.number(16), first = h.number(16), last = h.number(16);
            if (zid == 0) continue;
            int64_t bc = h.number(16), ftype = h.number(16);
            if (!h.ends_with_paren()) {
                const char *b, *e;
                c.line(b, e);
            }
            Zone &z = m.zones[m.zone_slot(zid)];
            z.first = first;
            z.last = last;
            z.bc = bc;
            z.size = last - first + 1;
            int64_t cnt = z.size;
            m.face_c0.reserve(m.face_c0.size() + cnt);
            m.face_c1.reserve(m.face_c1.size() + cnt);
            for (int64_t i = 0; i < cnt; ++i) {
                int64_t t = ftype;
                if (ftype == 0 && !c.hex(t)) fmt("truncated face section");
                if (t != 2 && t != 3 && t != 4) raise(PSST_ERR_FORMAT, "Error: Unknown face type!");
                for (int64_t j = 0; j < t; ++j) {
                    int64_t v;
                    if (!c.hex(v)) fmt("truncated face section");
                    m.face_nodes.push_back(v);
                }
                int64_t c0, c1;
                if (!c.hex(c0) || !c.hex(c1)) fmt("truncated face section");
                // read_faces hands (c1, c0) to add_face(left, right) and the face
                // stores cell(0) = right, cell(1) = left
                // (psstAnsysGridReader.cpp:1026, :192-193): file order is kept.
                m.face_c0.push_back(c0);
                m.face_c1.push_back(c1);
                m.face_ptr.push_back((int64_t)m.face_nodes.size());
            }
        } else if (op == 39 || op == 45) {
            int64_t zid = h.number(10);
            h.name();
            std::string name = h.name();
            m.zones[m.zone_slot(zid)].name = name;
        } else if (op == 58 || op == 59) {
            // cell/face trees of adapted meshes (read_cell_tree / read_face_tree,
            // psstAnsysGridReader.cpp:1068-1116): kept for the case writer; no step
            // of the loop reads them. A parent zone no section declared gets bc 31
            // (add_zones_storage_connection, :655-686).
            RawMesh::Tree t;
            t.op = (int)op;
            t.first = h.number(16);
            t.last = h.number(16);
            t.parent_zone = h.number(16);
            t.child_zone = h.number(16);
            if (!h.ends_with_paren()) {
                const char *b, *e;
                c.line(b, e);
            }
            bool known = false;
            for (const Zone &z : m.zones) known = known || z.id == t.parent_zone;
            if (!known) {
                Zone &z = m.zones[m.zone_slot(t.parent_zone)];
                z.first = t.first;
                z.last = t.last;
                z.bc = 31;
                z.size = t.last - t.first + 1;
            }
            t.ptr.push_back(0);
            for (int64_t i = 0; i < t.last - t.first + 1; ++i) {
                int64_t nk, kid;
                if (!c.hex(nk)) fmt("truncated tree section");
                for (int64_t j = 0; j < nk; ++j) {
                    if (!c.hex(kid)) fmt("truncated tree section");
                    t.kids.push_back(kid);
                }
                t.ptr.push_back((int64_t)t.kids.size());
            }
            m.trees.push_back(std::move(t));
        }
    }
    if (m.dim != 2 && m.dim != 3) fmt("missing or invalid dimension section");
    return m;
}

}  // namespace psst
