// The reference's YAML operator format (README:27-187, yaml.cpp:169-271): a
// list of unique MPO sites and a 1-based `sequence` that orders them into the
// chain.  Host-only; no yaml-cpp: the YAML subset the format uses is parsed
// here (block mappings and sequences by indentation, compact "- key: value"
// items, flow sequences and mappings, plain and quoted scalars, comments,
// document markers, anchors &name and aliases *name).
//
//   sites:
//     - physical dimension: 2
//       left dimension:     1
//       right dimension:    3
//       matrices:
//         - from: 1
//           to:   2
//           data: [0,1,1,0]          # d*d entries, row-major as written
//   sequence: [1, 2, 2, 3]
//
// Complex entries are a scalar (real), a [re, im] pair or {real: re, imag: im}
// (yaml.hpp:55-69).  The data list is stored as written into the (d,d)
// column-major block of the site, i.e. W(o1,o2) = M[o2][o1].  Errors carry the
// reference's messages (yaml.cpp:47-76, io.hpp:100-160).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nutcracker_b200.h"
#include "nc_parsed_operator.h"

using nc::g_status;

namespace {

struct YNode;
using YPtr = std::shared_ptr<const YNode>;

struct YNode {
    enum Kind { Null, Scalar, Seq, Map } kind = Null;
    std::string scalar;
    std::vector<YPtr> seq;
    std::vector<std::pair<std::string, YPtr>> map;
    const YNode* get(const std::string& key) const {
        if (kind != Map) return nullptr;
        for (const auto& kv : map)
            if (kv.first == key) return kv.second.get();
        return nullptr;
    }
    size_t size() const { return kind == Seq ? seq.size() : kind == Map ? map.size() : 0; }
};

[[noreturn]] void fail(const std::string& msg) { throw nc::Error(nc::NC_ERR_ARG, msg); }

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r')) ++a;
    while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r')) --b;
    return s.substr(a, b - a);
}

struct Line {
    int indent;
    std::string text;   // content after the indentation, comment removed
    int number;         // 1-based line number in the document
};

// Position of a top-level "key:" separator (':' followed by a space or the end
// of the text, outside quotes and brackets), or npos.
size_t key_separator(const std::string& s) {
    int depth = 0;
    char quote = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (quote) {
            if (c == quote) quote = 0;
            continue;
        }
        if (c == '"' || c == '\'') quote = c;
        else if (c == '[' || c == '{') ++depth;
        else if (c == ']' || c == '}') --depth;
        else if (c == ':' && depth == 0 && (i + 1 == s.size() || s[i + 1] == ' ' || s[i + 1] == '\t'))
            return i;
    }
    return std::string::npos;
}

std::string strip_comment(const std::string& s) {
    char quote = 0;
    for (size_t i = 0; i < s.size(); ++i) {
        const char c = s[i];
        if (quote) {
            if (c == quote) quote = 0;
            continue;
        }
        if (c == '"' || c == '\'') quote = c;
        else if (c == '#' && (i == 0 || s[i - 1] == ' ' || s[i - 1] == '\t')) return s.substr(0, i);
    }
    return s;
}

bool is_seq_item(const std::string& t) { return t == "-" || (t.size() > 1 && t[0] == '-' && (t[1] == ' ' || t[1] == '\t')); }

class Parser {
  public:
    explicit Parser(const std::string& text) {
        size_t pos = 0;
        int number = 0;
        bool started = false;
        while (pos <= text.size()) {
            size_t end = text.find('\n', pos);
            if (end == std::string::npos) end = text.size();
            std::string raw = text.substr(pos, end - pos);
            pos = end + 1;
            ++number;
            const size_t first = raw.find_first_not_of(" \t\r");
            if (first != std::string::npos && raw.substr(0, first).find('\t') != std::string::npos)
                fail("YAML: tab used for indentation on line " + std::to_string(number));
            std::string body = strip_comment(raw);
            const std::string t = trim(body);
            if (t.empty()) continue;
            if (t.compare(0, 3, "---") == 0 && (t.size() == 3 || t[3] == ' ')) {
                if (started || !lines_.empty()) break;   // the first document only
                started = true;
                const std::string rest = trim(t.substr(3));
                if (!rest.empty()) lines_.push_back({0, rest, number});
                continue;
            }
            if (t == "...") break;
            const int indent = (int)body.find_first_not_of(' ');
            lines_.push_back({indent, trim(body.substr(indent)), number});
            if (pos > text.size()) break;
        }
    }

    YPtr document() {
        size_t i = 0;
        if (lines_.empty()) return std::make_shared<YNode>();
        YPtr root = block(i, lines_[0].indent);
        if (i < lines_.size()) fail("YAML: unexpected content on line " + std::to_string(lines_[i].number));
        return root;
    }

  private:
    std::vector<Line> lines_;
    std::map<std::string, YPtr> anchors_;
    // Nesting depth of the recursive descent; operator files nest a few
    // levels, and a bound keeps malformed input from exhausting the stack.
    static constexpr int kMaxDepth = 256;
    int depth_ = 0;
    struct Nest {
        int& d;
        Nest(int& depth, int number) : d(depth) {
            if (d >= kMaxDepth)
                fail("YAML: nesting deeper than " + std::to_string(kMaxDepth) + " levels on line " +
                     std::to_string(number));
            ++d;
        }
        ~Nest() { --d; }
    };

    YPtr block(size_t& i, int indent) {
        const Line& l = lines_[i];
        Nest nest(depth_, l.number);
        if (is_seq_item(l.text)) return sequence(i, l.indent);
        if (key_separator(l.text) != std::string::npos && l.text[0] != '[' && l.text[0] != '{')
            return mapping(i, l.indent);
        // a lone (possibly multi-line flow) value
        std::string v = l.text;
        ++i;
        while (!balanced(v) && i < lines_.size()) v += " " + lines_[i++].text;
        (void)indent;
        return inline_value(v, l.number);
    }

    // A value that continues on following lines: a nested block at a deeper
    // indentation, or a block sequence at the key's own indentation.
    YPtr child(size_t& i, int parent_indent, bool seq_at_same_indent) {
        if (i < lines_.size()) {
            const Line& n = lines_[i];
            if (n.indent > parent_indent) return block(i, n.indent);
            if (seq_at_same_indent && n.indent == parent_indent && is_seq_item(n.text)) return sequence(i, n.indent);
        }
        return std::make_shared<YNode>();
    }

    YPtr sequence(size_t& i, int indent) {
        auto node = std::make_shared<YNode>();
        node->kind = YNode::Seq;
        while (i < lines_.size() && lines_[i].indent == indent && is_seq_item(lines_[i].text)) {
            Line& l = lines_[i];
            size_t off = 1;
            while (off < l.text.size() && (l.text[off] == ' ' || l.text[off] == '\t')) ++off;
            const std::string rest = l.text.substr(off);
            if (rest.empty()) {
                ++i;
                node->seq.push_back(child(i, indent, false));
                continue;
            }
            std::string anchor;
            std::string body = rest;
            if (body[0] == '&') {   // "- &name" followed by a block, or "- &name value"
                const size_t sp = body.find(' ');
                anchor = body.substr(1, sp == std::string::npos ? std::string::npos : sp - 1);
                body = sp == std::string::npos ? std::string() : trim(body.substr(sp));
                if (body.empty()) {
                    ++i;
                    YPtr v = child(i, indent, false);
                    anchors_[anchor] = v;
                    node->seq.push_back(v);
                    continue;
                }
            }
            if (is_seq_item(body) || (key_separator(body) != std::string::npos && body[0] != '[' && body[0] != '{')) {
                // compact nested item: re-read this line as a block at the item's column
                l.indent = indent + (int)(l.text.size() - body.size());
                l.text = body;
                YPtr v = block(i, l.indent);
                if (!anchor.empty()) anchors_[anchor] = v;
                node->seq.push_back(v);
                continue;
            }
            std::string v = body;
            const int number = l.number;
            ++i;
            while (!balanced(v) && i < lines_.size()) v += " " + lines_[i++].text;
            YPtr val = inline_value(v, number);
            if (!anchor.empty()) anchors_[anchor] = val;
            node->seq.push_back(val);
        }
        return node;
    }

    YPtr mapping(size_t& i, int indent) {
        auto node = std::make_shared<YNode>();
        node->kind = YNode::Map;
        while (i < lines_.size() && lines_[i].indent == indent && !is_seq_item(lines_[i].text)) {
            const Line& l = lines_[i];
            const size_t sep = key_separator(l.text);
            if (sep == std::string::npos)
                fail("YAML: expected 'key: value' on line " + std::to_string(l.number));
            const std::string key = unquote(trim(l.text.substr(0, sep)));
            std::string value = trim(l.text.substr(sep + 1));
            const int number = l.number;
            ++i;
            std::string anchor;
            if (!value.empty() && value[0] == '&') {
                const size_t sp = value.find(' ');
                anchor = value.substr(1, sp == std::string::npos ? std::string::npos : sp - 1);
                value = sp == std::string::npos ? std::string() : trim(value.substr(sp));
            }
            YPtr v;
            if (value.empty()) {
                v = child(i, indent, true);
            } else {
                while (!balanced(value) && i < lines_.size()) value += " " + lines_[i++].text;
                v = inline_value(value, number);
            }
            if (!anchor.empty()) anchors_[anchor] = v;
            node->map.emplace_back(key, v);
        }
        return node;
    }

    static bool balanced(const std::string& s) {
        int depth = 0;
        char quote = 0;
        for (char c : s) {
            if (quote) {
                if (c == quote) quote = 0;
                continue;
            }
            if (c == '"' || c == '\'') quote = c;
            else if (c == '[' || c == '{') ++depth;
            else if (c == ']' || c == '}') --depth;
        }
        return depth <= 0;
    }

    static std::string unquote(const std::string& s) {
        if (s.size() >= 2 && (s[0] == '"' || s[0] == '\'') && s.back() == s[0]) return s.substr(1, s.size() - 2);
        return s;
    }

    YPtr inline_value(const std::string& text, int number) {
        size_t p = 0;
        YPtr v = flow(text, p, number);
        skip_ws(text, p);
        if (p != text.size()) fail("YAML: unexpected '" + text.substr(p) + "' on line " + std::to_string(number));
        return v;
    }

    static void skip_ws(const std::string& s, size_t& p) {
        while (p < s.size() && (s[p] == ' ' || s[p] == '\t')) ++p;
    }

    YPtr flow(const std::string& s, size_t& p, int number) {
        Nest nest(depth_, number);
        skip_ws(s, p);
        if (p < s.size() && s[p] == '&') {
            size_t e = p + 1;
            while (e < s.size() && s[e] != ' ' && s[e] != ',' && s[e] != ']' && s[e] != '}') ++e;
            const std::string name = s.substr(p + 1, e - p - 1);
            p = e;
            YPtr v = flow(s, p, number);
            anchors_[name] = v;
            return v;
        }
        if (p < s.size() && s[p] == '*') {
            size_t e = p + 1;
            while (e < s.size() && s[e] != ' ' && s[e] != ',' && s[e] != ']' && s[e] != '}') ++e;
            const std::string name = s.substr(p + 1, e - p - 1);
            p = e;
            auto it = anchors_.find(name);
            if (it == anchors_.end()) fail("YAML: unknown alias *" + name + " on line " + std::to_string(number));
            return it->second;
        }
        if (p < s.size() && s[p] == '[') {
            auto node = std::make_shared<YNode>();
            node->kind = YNode::Seq;
            ++p;
            skip_ws(s, p);
            if (p < s.size() && s[p] == ']') {
                ++p;
                return node;
            }
            for (;;) {
                node->seq.push_back(flow(s, p, number));
                skip_ws(s, p);
                if (p < s.size() && s[p] == ',') {
                    ++p;
                    continue;
                }
                if (p < s.size() && s[p] == ']') {
                    ++p;
                    return node;
                }
                fail("YAML: malformed flow sequence on line " + std::to_string(number));
            }
        }
        if (p < s.size() && s[p] == '{') {
            auto node = std::make_shared<YNode>();
            node->kind = YNode::Map;
            ++p;
            skip_ws(s, p);
            if (p < s.size() && s[p] == '}') {
                ++p;
                return node;
            }
            for (;;) {
                skip_ws(s, p);
                size_t e = p;
                while (e < s.size() && s[e] != ':') ++e;
                if (e >= s.size()) fail("YAML: malformed flow mapping on line " + std::to_string(number));
                const std::string key = unquote(trim(s.substr(p, e - p)));
                p = e + 1;
                node->map.emplace_back(key, flow(s, p, number));
                skip_ws(s, p);
                if (p < s.size() && s[p] == ',') {
                    ++p;
                    continue;
                }
                if (p < s.size() && s[p] == '}') {
                    ++p;
                    return node;
                }
                fail("YAML: malformed flow mapping on line " + std::to_string(number));
            }
        }
        // scalar: quoted, or plain up to a flow delimiter
        auto node = std::make_shared<YNode>();
        node->kind = YNode::Scalar;
        if (p < s.size() && (s[p] == '"' || s[p] == '\'')) {
            const char q = s[p];
            const size_t e = s.find(q, p + 1);
            if (e == std::string::npos) fail("YAML: unterminated string on line " + std::to_string(number));
            node->scalar = s.substr(p + 1, e - p - 1);
            p = e + 1;
            return node;
        }
        size_t e = p;
        while (e < s.size() && s[e] != ',' && s[e] != ']' && s[e] != '}') ++e;
        node->scalar = trim(s.substr(p, e - p));
        if (node->scalar == "~" || node->scalar == "null") node->kind = YNode::Null;
        p = e;
        return node;
    }
};

double as_double(const YNode* n, const char* what) {
    if (!n || n->kind != YNode::Scalar) fail(std::string("YAML: ") + what + " must be a number");
    const char* s = n->scalar.c_str();
    char* end = nullptr;
    const double v = std::strtod(s, &end);
    if (end == s || *end != '\0') fail(std::string("YAML: bad number '") + n->scalar + "' for " + what);
    return v;
}

long long as_integer(const YNode* n, const char* what) {
    if (!n || n->kind != YNode::Scalar) fail(std::string("YAML: missing or non-scalar '") + what + "'");
    const char* s = n->scalar.c_str();
    char* end = nullptr;
    const long long v = std::strtoll(s, &end, 10);
    if (end == s || *end != '\0') fail(std::string("YAML: bad integer '") + n->scalar + "' for '" + what + "'");
    return v;
}

nc_complex as_complex(const YNode* n) {
    nc_complex z;
    z.re = 0;
    z.im = 0;
    if (!n) fail("YAML: missing matrix entry");
    if (n->kind == YNode::Scalar) {
        z.re = as_double(n, "a matrix entry");
    } else if (n->kind == YNode::Seq && n->seq.size() == 2) {
        z.re = as_double(n->seq[0].get(), "a matrix entry");
        z.im = as_double(n->seq[1].get(), "a matrix entry");
    } else if (n->kind == YNode::Map) {
        z.re = as_double(n->get("real"), "a matrix entry");
        z.im = as_double(n->get("imag"), "a matrix entry");
    } else {
        fail("YAML: bad node type for complex number");
    }
    return z;
}

std::string fmt(const char* f, long long a) {
    char b[256];
    std::snprintf(b, sizeof b, f, a);
    return b;
}

using UniqueSite = nc_parsed_operator::Site;

// OperatorSite reader (yaml.cpp:217-256).
UniqueSite read_site(const YNode& node) {
    UniqueSite s;
    const long long d = as_integer(node.get("physical dimension"), "physical dimension");
    const long long cl = as_integer(node.get("left dimension"), "left dimension");
    const long long cr = as_integer(node.get("right dimension"), "right dimension");
    if (d < 1 || cl < 1 || cr < 1) fail("YAML: site dimensions must be positive");
    // the dimensions are unsigned 32-bit integers in the operator format
    if (d > UINT32_MAX || cl > UINT32_MAX || cr > UINT32_MAX)
        fail("YAML: site dimensions must be below 2^32");
    s.d = (uint32_t)d;
    s.cl = (uint32_t)cl;
    s.cr = (uint32_t)cr;
    const YNode* mats = node.get("matrices");
    const size_t nnz = mats ? mats->size() : 0;
    const size_t len = (size_t)d * d;
    for (size_t k = 0; k < nnz; ++k) {
        const YNode* m = mats->kind == YNode::Seq ? mats->seq[k].get() : mats->map[k].second.get();
        const long long from = as_integer(m->get("from"), "from");
        if (from < 1) fail(fmt("The 'from' index is too low. (%lld < 1)", from));
        if (from > cl)
            fail(fmt("The 'from' index is too high. (%lld > ", from) + std::to_string(cl) + ")");
        const long long to = as_integer(m->get("to"), "to");
        if (to < 1) fail(fmt("The 'to' index is too low. (%lld < 1)", to));
        if (to > cr) fail(fmt("The 'to' index is too high. (%lld > ", to) + std::to_string(cr) + ")");
        s.idx.push_back((uint32_t)from);
        s.idx.push_back((uint32_t)to);
        const YNode* data = m->get("data");
        const size_t n = data ? data->size() : 0;
        if (!data || data->kind != YNode::Seq || n != len)
            fail(fmt("The length of the data (%lld) does not match the correct length (", (long long)n) +
                 std::to_string(len) + ").");
        for (size_t e = 0; e < len; ++e) s.W.push_back(as_complex(data->seq[e].get()));
    }
    return s;
}

}  // namespace

void nc_parsed_operator::assemble() {
    // constructOperatorFrom (io.hpp:350-370)
    if (sequence.empty()) fail("No operator sites were specified.");
    for (size_t k = 0; k < sequence.size(); ++k) {
        const uint32_t index = sequence[k];
        if (index >= unique.size())
            fail(fmt("When reading in an operator, a reference to the non-existent operator site number %lld "
                     "appeared in the sequence.", (long long)index));
        const UniqueSite& u = unique[index];
        if (k == 0) {
            if (u.cl != 1) fail(fmt("The left dimension of the left-most site must be one but instead is %lld.", u.cl));
        } else {
            const UniqueSite& prev = unique[sequence[k - 1]];
            if (u.cl != prev.cr) {
                char b[256];
                std::snprintf(b, sizeof b,
                              "The left dimension (%u) of site %zu does not match the right dimension (%u) of site "
                              "%zu.  (%u != %u)",
                              u.cl, k - 1, prev.cr, k, u.cl, prev.cr);
                fail(b);
            }
        }
    }
    const UniqueSite& last = unique[sequence.back()];
    if (last.cr != 1) fail(fmt("The right dimension of the right-most site must be one but instead is %lld.", last.cr));
    sites.clear();
    for (uint32_t index : sequence) {
        const UniqueSite& u = unique[index];
        nc_operator_site s;
        s.physical_dimension = u.d;
        s.left_dimension = u.cl;
        s.right_dimension = u.cr;
        s.number_of_matrices = (uint32_t)(u.idx.size() / 2);
        s.indices = u.idx.data();
        s.matrices = u.W.data();
        sites.push_back(s);
    }
}

extern "C" {

nc_parsed_operator* nc_yaml_read_operator(const char* text, size_t length, const char* location) {
    NC_ABI_BEGIN
    NC_ARG(text != nullptr, "nc_yaml_read_operator: null text");
    Parser parser(std::string(text, length));
    YPtr root = parser.document();
    const YNode* node = root.get();
    if (location && *location) {
        // slash-separated keys (LocationSlashTokenizer, io.hpp:344-346)
        std::string loc(location), part;
        size_t p = 0;
        while (p <= loc.size()) {
            size_t e = loc.find('/', p);
            if (e == std::string::npos) e = loc.size();
            part = loc.substr(p, e - p);
            p = e + 1;
            if (part.empty()) continue;
            node = node ? node->get(part) : nullptr;
            if (!node) fail("No such location " + loc + ".");
        }
    }
    auto op = std::make_unique<nc_parsed_operator>();
    const YNode* sites = node ? node->get("sites") : nullptr;
    if (sites && sites->kind == YNode::Seq)
        for (const YPtr& s : sites->seq) {
            if (!s || s->kind != YNode::Map) fail("YAML: every entry of 'sites' must be a mapping");
            op->unique.push_back(read_site(*s));
        }
    else if (sites && sites->kind != YNode::Null)
        fail("YAML: 'sites' must be a list");
    const YNode* seq = node ? node->get("sequence") : nullptr;
    if (seq && seq->kind == YNode::Seq)
        for (const YPtr& e : seq->seq) op->sequence.push_back((uint32_t)(as_integer(e.get(), "sequence") - 1));
    op->assemble();
    return op.release();
    NC_ABI_END
    return nullptr;
}

uint32_t nc_parsed_operator_number_of_sites(const nc_parsed_operator* op) { return op ? (uint32_t)op->sites.size() : 0; }

const nc_operator_site* nc_parsed_operator_sites(const nc_parsed_operator* op) {
    return op && !op->sites.empty() ? op->sites.data() : nullptr;
}

void nc_parsed_operator_free(nc_parsed_operator* op) { delete op; }

size_t nc_yaml_write_operator(uint32_t number_of_sites, const nc_operator_site* sites, char* out, size_t capacity) {
    // Operator emitter (yaml.cpp:186-206, 257-306): unique sites (here by
    // content) and the 1-based sequence; entries with a zero imaginary part
    // are written as reals, others as [re, im], with 20 significant digits.
    std::string s;
    std::vector<const nc_operator_site*> unique;
    std::vector<uint32_t> sequence;
    auto same = [](const nc_operator_site* a, const nc_operator_site* b) {
        if (a->physical_dimension != b->physical_dimension || a->left_dimension != b->left_dimension ||
            a->right_dimension != b->right_dimension || a->number_of_matrices != b->number_of_matrices)
            return false;
        const size_t nnz = a->number_of_matrices, dd = (size_t)a->physical_dimension * a->physical_dimension;
        return std::memcmp(a->indices, b->indices, sizeof(uint32_t) * 2 * nnz) == 0 &&
               std::memcmp(a->matrices, b->matrices, sizeof(nc_complex) * dd * nnz) == 0;
    };
    for (uint32_t i = 0; i < number_of_sites; ++i) {
        uint32_t k = 0;
        while (k < unique.size() && !same(unique[k], &sites[i])) ++k;
        if (k == unique.size()) unique.push_back(&sites[i]);
        sequence.push_back(k + 1);
    }
    auto num = [](double x) {
        char b[64];
        std::snprintf(b, sizeof b, "%.20g", x);
        return std::string(b);
    };
    s += "sequence: [";
    for (size_t i = 0; i < sequence.size(); ++i) s += (i ? ", " : "") + std::to_string(sequence[i]);
    s += "]\nsites:\n";
    for (const nc_operator_site* u : unique) {
        s += "  - physical dimension: " + std::to_string(u->physical_dimension) + "\n";
        s += "    left dimension: " + std::to_string(u->left_dimension) + "\n";
        s += "    right dimension: " + std::to_string(u->right_dimension) + "\n";
        s += "    matrices:\n";
        const size_t dd = (size_t)u->physical_dimension * u->physical_dimension;
        for (uint32_t k = 0; k < u->number_of_matrices; ++k) {
            s += "      - from: " + std::to_string(u->indices[2 * k]) + "\n";
            s += "        to: " + std::to_string(u->indices[2 * k + 1]) + "\n";
            s += "        data: [";
            for (size_t e = 0; e < dd; ++e) {
                const nc_complex z = u->matrices[k * dd + e];
                if (e) s += ", ";
                s += z.im == 0 ? num(z.re) : "[" + num(z.re) + ", " + num(z.im) + "]";
            }
            s += "]\n";
        }
    }
    if (out && capacity > 0) {
        const size_t n = std::min(capacity - 1, s.size());
        std::memcpy(out, s.data(), n);
        out[n] = '\0';
    }
    return s.size();
}

}  // extern "C"
