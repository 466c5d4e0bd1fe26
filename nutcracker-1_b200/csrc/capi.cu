// C API with the reference's names (include/nutcracker.h; sources/c-interface/*.cpp):
// matrices, vectors, operator and state terms, the builders with their
// automaton compiler (compiler.hpp:419-938, compiler.cpp), protobuf
// serialization (nutcracker.proto, protobuf.cpp) and the simple solvers.
//
// The compiler is host code: a builder collects, per site, the transitions
// (left signal, right signal) -> matrix of a finite automaton whose paths from
// the start signal 1 to the end signal 2 spell the terms of the operator;
// optimisation removes null transitions and dead signals and merges signals
// with identical incoming (or outgoing) transitions, and compilation numbers
// each site's signals into MPO bond indices.  Solves and state contractions
// run on the GPU through the library's chain and Level-0 kernels.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "nc_abi_util.h"
#include "nc_common.cuh"
#include "nc_parsed_operator.h"
#include "nutcracker.h"
#include "nutcracker_b200.h"

namespace {

using cd = std::complex<double>;

thread_local std::unique_ptr<std::string> t_error;

void set_error(const std::string& m) { t_error.reset(new std::string(m)); }

#define C_BEGIN try {
#define C_END(ret)                          \
    }                                       \
    catch (const std::exception& e) {       \
        set_error(e.what());                \
        return ret;                         \
    }                                       \
    catch (...) {                           \
        set_error("unknown error");         \
        return ret;                         \
    }

// ---------------------------------------------------------------------------
// dense data: square matrices (row-major) and vectors
// ---------------------------------------------------------------------------
struct Data {
    uint32_t n = 0;          // matrix dimension, or vector length
    bool matrix = true;
    std::vector<cd> a;       // n*n (row-major) or n entries
};
using DataPtr = std::shared_ptr<const Data>;

DataPtr make_matrix(uint32_t n, const cd* row_major) {
    auto d = std::make_shared<Data>();
    d->n = n;
    d->a.assign(row_major, row_major + (size_t)n * n);
    return d;
}
DataPtr make_vector(uint32_t n, const cd* v) {
    auto d = std::make_shared<Data>();
    d->n = n;
    d->matrix = false;
    d->a.assign(v, v + n);
    return d;
}
DataPtr scaled(const DataPtr& x, cd c) {
    auto d = std::make_shared<Data>(*x);
    for (cd& v : d->a) v *= c;
    return d;
}
DataPtr summed(const DataPtr& x, const DataPtr& y) {
    if (x->n != y->n || x->matrix != y->matrix)
        throw std::logic_error("Cannot add objects of different dimensions (" + std::to_string(x->n) + " != " +
                               std::to_string(y->n) + ").");
    auto d = std::make_shared<Data>(*x);
    for (size_t i = 0; i < d->a.size(); ++i) d->a[i] += y->a[i];
    return d;
}
DataPtr identity(uint32_t n) {
    std::vector<cd> a((size_t)n * n, cd(0, 0));
    for (uint32_t i = 0; i < n; ++i) a[(size_t)i * n + i] = 1;
    return make_matrix(n, a.data());
}

// Table of distinct non-null data; id 0 is the null entry (DataTable,
// compiler.hpp:108-246): entries within 1e-14 of each other share an id.
class DataTable {
  public:
    DataTable() { store_.emplace_back(); }
    const DataPtr& get(unsigned id) const { return store_[id]; }
    unsigned lookup(const DataPtr& d) {
        if (d->n == 0) return 0;
        bool null = true;
        for (const cd& v : d->a)
            if (std::abs(v) >= 1e-14) null = false;
        if (null) return 0;
        for (unsigned id = 1; id < store_.size(); ++id) {
            const Data& e = *store_[id];
            if (e.n != d->n || e.matrix != d->matrix) continue;
            bool same = true;
            for (size_t i = 0; i < e.a.size() && same; ++i) same = std::abs(e.a[i] - d->a[i]) <= 1e-14;
            if (same) return id;
        }
        store_.push_back(d);
        return (unsigned)store_.size() - 1;
    }
    unsigned lookup_sum(const std::vector<unsigned>& ids) {
        if (ids.empty()) return 0;
        if (ids.size() == 1) return ids[0];
        DataPtr total = get(ids[0]);
        for (size_t k = 1; k < ids.size(); ++k) total = summed(total, get(ids[k]));
        return lookup(total);
    }

  private:
    std::vector<DataPtr> store_;
};

constexpr unsigned kStart = 1, kEnd = 2;
using Key = std::pair<unsigned, unsigned>;        // (left signal, right signal)
using SiteConnections = std::map<Key, unsigned>;  // -> data id

unsigned in_sig(bool fwd, const Key& k) { return fwd ? k.first : k.second; }
unsigned out_sig(bool fwd, const Key& k) { return fwd ? k.second : k.first; }
Key make_key(bool fwd, unsigned in, unsigned out) { return fwd ? Key(in, out) : Key(out, in); }

std::string set_string(const std::set<unsigned>& s) {
    std::ostringstream o;
    o << '[';
    bool first = true;
    for (unsigned v : s) {
        if (!first) o << ',';
        first = false;
        o << v;
    }
    o << ']';
    return o.str();
}

}  // namespace

namespace {

// One compiled site: an MPO site (idx (2,nnz) 1-based, W (d,d,nnz) column-major
// with W(o1,o2) = M[o2][o1]) or an MPS site (A (br,bl,d) column-major).
struct SiteData {
    uint32_t d = 0, cl = 0, cr = 0;
    std::vector<uint32_t> idx;
    std::vector<nc_complex> W;
};
using SitePtr = std::shared_ptr<const SiteData>;

struct Link {
    unsigned from, to;
    DataPtr data;
};

// constructOperatorSite (operators.cpp:83-112)
SiteData operator_site(uint32_t d, uint32_t cl, uint32_t cr, const std::vector<Link>& links) {
    SiteData s;
    s.d = d;
    s.cl = cl;
    s.cr = cr;
    for (const Link& l : links) {
        s.idx.push_back(l.from);
        s.idx.push_back(l.to);
        const Data& m = *l.data;
        for (uint32_t o2 = 0; o2 < d; ++o2)
            for (uint32_t o1 = 0; o1 < d; ++o1) {
                const cd v = m.a[(size_t)o2 * d + o1];   // M[o2][o1]
                s.W.push_back(nc_complex{v.real(), v.imag()});
            }
    }
    return s;
}

// constructStateSite (states.cpp:30-62): link (from, to) holds the vector
// over the physical index at (to-1) + (from-1)*br, stride bl*br.
SiteData state_site(uint32_t d, uint32_t cl, uint32_t cr, const std::vector<Link>& links) {
    SiteData s;
    s.d = d;
    s.cl = cl;
    s.cr = cr;
    s.W.assign((size_t)d * cl * cr, nc_complex{0, 0});
    for (const Link& l : links)
        for (uint32_t o = 0; o < d; ++o) {
            const cd v = l.data->a[o];
            s.W[(size_t)(l.to - 1) + (size_t)(l.from - 1) * cr + (size_t)o * cl * cr] = nc_complex{v.real(), v.imag()};
        }
    return s;
}

// The automaton of one operator or state (Specification, compiler.hpp:444-695).
class Specification {
  public:
    DataTable table;
    std::vector<SiteConnections> connections;
    unsigned next_free_signal = 3;

    unsigned allocate_signal() { return next_free_signal++; }
    void connect(unsigned site, unsigned from, unsigned to, unsigned id) {
        if (connections.size() <= site) connections.resize(site + 1);
        connections[site][Key(from, to)] = id;
    }

    void optimize() {
        for (bool go = true; go; go = eliminate_null() || eliminate_dead(true, kStart) || eliminate_dead(false, kEnd) ||
                                      merge(true) || merge(false)) {
        }
    }

    // Sites with their signals numbered 1.. in signal order (compile,
    // compiler.hpp:469-531); `make` builds one site from its links.
    template <typename Make>
    std::vector<SitePtr> compile(Make make) const {
        std::vector<SitePtr> sites;
        std::map<unsigned, unsigned> left_map{{kStart, 1}};
        unsigned site_number = 0;
        std::map<std::vector<std::tuple<unsigned, unsigned, const Data*>>, SitePtr> index;
        for (const SiteConnections& sc : connections) {
            std::set<unsigned> lefts, rights, expected;
            for (const auto& kv : sc) {
                lefts.insert(kv.first.first);
                rights.insert(kv.first.second);
            }
            for (const auto& kv : left_map) expected.insert(kv.first);
            if (lefts != expected) conflict(site_number, expected, lefts);
            std::map<unsigned, unsigned> right_map;
            unsigned next = 1;
            for (unsigned r : rights) right_map[r] = next++;
            std::vector<Link> links;
            std::vector<std::tuple<unsigned, unsigned, const Data*>> key;
            for (const auto& kv : sc) {
                links.push_back(Link{left_map[kv.first.first], right_map[kv.first.second], table.get(kv.second)});
                key.emplace_back(links.back().from, links.back().to, links.back().data.get());
            }
            auto it = index.find(key);
            SitePtr site;
            if (it != index.end()) {
                site = it->second;
            } else {
                if (links.empty()) throw std::logic_error("site " + std::to_string(site_number) + " has no terms");
                site = std::make_shared<SiteData>(make(links[0].data->n, (uint32_t)lefts.size(), (uint32_t)rights.size(), links));
                index[key] = site;
            }
            sites.push_back(site);
            ++site_number;
            left_map = right_map;
        }
        std::set<unsigned> last, end{kEnd};
        for (const auto& kv : left_map) last.insert(kv.first);
        if (last != end) conflict(site_number, last, end);
        return sites;
    }

  private:
    [[noreturn]] static void conflict(unsigned site, const std::set<unsigned>& left_site_right,
                                      const std::set<unsigned>& right_site_left) {
        throw std::logic_error("The left signals at site " + std::to_string(site) + ", " + set_string(right_site_left) +
                               ", do not match the right signals of its left neighbor, " +
                               set_string(left_site_right) + ".");
    }

    bool eliminate_null() {
        bool changed = false;
        for (SiteConnections& sc : connections)
            for (auto it = sc.begin(); it != sc.end();) {
                if (it->second == 0) {
                    it = sc.erase(it);
                    changed = true;
                } else {
                    ++it;
                }
            }
        return changed;
    }

    // Transitions unreachable from the start (forward) or that cannot reach
    // the end (backward) are removed.
    bool eliminate_dead(bool fwd, unsigned first) {
        bool changed = false;
        std::set<unsigned> incoming{first};
        const size_t n = connections.size();
        for (size_t k = 0; k < n; ++k) {
            SiteConnections& sc = connections[fwd ? k : n - 1 - k];
            std::set<unsigned> outgoing;
            for (auto it = sc.begin(); it != sc.end();) {
                if (!incoming.count(in_sig(fwd, it->first))) {
                    it = sc.erase(it);
                    changed = true;
                } else {
                    outgoing.insert(out_sig(fwd, it->first));
                    ++it;
                }
            }
            incoming = outgoing;
        }
        return changed;
    }

    // Outgoing signals with identical incoming transitions become one signal;
    // the neighbour's transitions from them are summed (mergeSignalsGeneric).
    bool merge(bool fwd) {
        bool changed = false;
        const size_t n = connections.size();
        for (size_t k = 0; k + 1 < n; ++k) {
            SiteConnections& sc = connections[fwd ? k : n - 1 - k];
            SiteConnections& next = connections[fwd ? k + 1 : n - 2 - k];
            std::map<unsigned, std::map<unsigned, unsigned>> out_to_in;
            for (const auto& kv : sc) out_to_in[out_sig(fwd, kv.first)][in_sig(fwd, kv.first)] = kv.second;
            std::map<std::map<unsigned, unsigned>, std::vector<unsigned>> groups;
            for (const auto& kv : out_to_in) groups[kv.second].push_back(kv.first);
            for (const auto& g : groups) {
                const std::vector<unsigned>& outs = g.second;
                if (outs.size() <= 1) continue;
                changed = true;
                const unsigned merged = allocate_signal();
                for (const auto& in_id : g.first) {
                    for (unsigned o : outs) sc.erase(make_key(fwd, in_id.first, o));
                    sc[make_key(fwd, in_id.first, merged)] = in_id.second;
                }
                std::vector<Key> remove;
                std::map<unsigned, std::vector<unsigned>> sums;
                for (unsigned o : outs)
                    for (const auto& kv : next)
                        if (in_sig(fwd, kv.first) == o) {
                            remove.push_back(kv.first);
                            sums[out_sig(fwd, kv.first)].push_back(kv.second);
                        }
                for (const Key& key : remove) next.erase(key);
                for (const auto& s : sums) next[make_key(fwd, merged, s.first)] = table.lookup_sum(s.second);
            }
        }
        return changed;
    }
};

}  // namespace

namespace {

// Builder (compiler.hpp:780-901): per site, the (left, right) transitions of
// the terms added so far, each a list of data summed at specification time.
class Builder {
  public:
    Builder(std::vector<uint32_t> dims, bool matrices) : dims_(std::move(dims)), matrices_(matrices), conn_(dims_.size()) {}
    unsigned number_of_sites() const { return (unsigned)dims_.size(); }
    unsigned dimension_of_site(unsigned s) const {
        if (s >= dims_.size()) site_too_large(s);
        return dims_[s];
    }
    unsigned allocate_signal() { return next_free_signal_++; }

    void connect(unsigned site, unsigned from, unsigned to, const DataPtr& data) {
        if (site >= dims_.size()) site_too_large(site);
        if (data->matrix != matrices_) throw std::logic_error("wrong kind of data for this builder");
        if (data->n != dims_[site])
            throw std::logic_error("Attempted to add matrix which has dimension " + std::to_string(data->n) +
                                   " to site number " + std::to_string(site) + " which has dimension " +
                                   std::to_string(dims_[site]) + ". (" + std::to_string(data->n) +
                                   " != " + std::to_string(dims_[site]) + ")");
        conn_[site][Key(from, to)].push_back(data);
    }

    void add_product_term(const std::vector<DataPtr>& components) {
        const unsigned n = number_of_sites();
        if (components.size() != n)
            throw std::logic_error("The number of sites in the argument (" + std::to_string(components.size()) +
                                   ") does not match the number of sites in the system (" + std::to_string(n) +
                                   ").  [" + std::to_string(components.size()) + " != " + std::to_string(n) + "]");
        if (n == 1) {
            connect(0, kStart, kEnd, components[0]);
            return;
        }
        const unsigned s = allocate_signal();
        connect(0, kStart, s, components[0]);
        for (unsigned i = 1; i + 1 < n; ++i) connect(i, s, s, components[i]);
        connect(n - 1, s, kEnd, components[n - 1]);
    }

    // generateSpecification (compiler.hpp:857-880, compiler.cpp:22-33)
    Specification specification(bool start_and_end_loops) const {
        Specification spec;
        spec.next_free_signal = std::max(spec.next_free_signal, next_free_signal_);
        spec.connections.resize(dims_.size());
        for (unsigned site = 0; site < dims_.size(); ++site)
            for (const auto& kv : conn_[site]) {
                DataPtr total = kv.second[0];
                for (size_t k = 1; k < kv.second.size(); ++k) total = summed(total, kv.second[k]);
                spec.connect(site, kv.first.first, kv.first.second, spec.table.lookup(total));
            }
        if (start_and_end_loops)
            for (unsigned site = 0; site < dims_.size(); ++site) {
                const unsigned id = spec.table.lookup(identity(dims_[site]));
                spec.connect(site, kStart, kStart, id);
                spec.connect(site, kEnd, kEnd, id);
            }
        return spec;
    }

  private:
    [[noreturn]] void site_too_large(unsigned s) const {
        throw std::logic_error("Site number " + std::to_string(s) + " is too large because there are only " +
                               std::to_string(dims_.size()) + " sites.");
    }
    std::vector<uint32_t> dims_;
    bool matrices_;
    std::vector<std::map<Key, std::vector<DataPtr>>> conn_;
    unsigned next_free_signal_ = 3;
};

// Terms (compiler.hpp:974-1141 and the C interface's wrappers, terms.hpp).
struct Term {
    virtual ~Term() {}
    virtual void apply(Builder& b) const = 0;
    virtual void multiply_by(cd c) = 0;
    virtual Term* copy() const = 0;
};

struct SumTerm : Term {
    std::unique_ptr<Term> a, b;
    SumTerm(const Term* x, const Term* y) : a(x->copy()), b(y->copy()) {}
    void apply(Builder& bl) const override {
        a->apply(bl);
        b->apply(bl);
    }
    // c (x + y) = c x + c y (the reference scales only its first summand)
    void multiply_by(cd c) override {
        a->multiply_by(c);
        b->multiply_by(c);
    }
    Term* copy() const override { return new SumTerm(a.get(), b.get()); }
};

struct LocalExternalField : Term {
    unsigned site;
    DataPtr field;
    LocalExternalField(unsigned s, DataPtr f) : site(s), field(std::move(f)) {}
    void apply(Builder& b) const override { b.connect(site, kStart, kEnd, field); }
    void multiply_by(cd c) override { field = scaled(field, c); }
    Term* copy() const override { return new LocalExternalField(*this); }
};

struct GlobalExternalField : Term {
    DataPtr field;
    explicit GlobalExternalField(DataPtr f) : field(std::move(f)) {}
    void apply(Builder& b) const override {
        for (unsigned s = 0; s < b.number_of_sites(); ++s) b.connect(s, kStart, kEnd, field);
    }
    void multiply_by(cd c) override { field = scaled(field, c); }
    Term* copy() const override { return new GlobalExternalField(*this); }
};

struct LocalNeighborCouplingField : Term {
    unsigned left_site;
    DataPtr left, right;
    LocalNeighborCouplingField(unsigned s, DataPtr l, DataPtr r) : left_site(s), left(std::move(l)), right(std::move(r)) {}
    void apply(Builder& b) const override {
        const unsigned s = b.allocate_signal();
        b.connect(left_site, kStart, s, left);
        b.connect(left_site + 1, s, kEnd, right);
    }
    void multiply_by(cd c) override { left = scaled(left, c); }
    Term* copy() const override { return new LocalNeighborCouplingField(*this); }
};

struct GlobalNeighborCouplingField : Term {
    DataPtr left, right;
    GlobalNeighborCouplingField(DataPtr l, DataPtr r) : left(std::move(l)), right(std::move(r)) {}
    void apply(Builder& b) const override {
        const unsigned s = b.allocate_signal();
        for (unsigned i = 0; i < b.number_of_sites(); ++i) {
            b.connect(i, kStart, s, left);
            b.connect(i, s, kEnd, right);
        }
    }
    void multiply_by(cd c) override { left = scaled(left, c); }
    Term* copy() const override { return new GlobalNeighborCouplingField(*this); }
};

struct ProductWithOneSiteDifferent : Term {
    unsigned site;
    DataPtr common, special;
    ProductWithOneSiteDifferent(unsigned s, DataPtr c, DataPtr sp) : site(s), common(std::move(c)), special(std::move(sp)) {}
    void apply(Builder& b) const override {
        if (site >= b.number_of_sites())
            throw std::logic_error("Site number " + std::to_string(site) + " is too large because there are only " +
                                   std::to_string(b.number_of_sites()) + " sites.");
        std::vector<DataPtr> comps(b.number_of_sites(), common);
        comps[site] = special;
        b.add_product_term(comps);
    }
    void multiply_by(cd c) override { special = scaled(special, c); }
    Term* copy() const override { return new ProductWithOneSiteDifferent(*this); }
};

// W state: sum over sites of the product with one site `special`.
struct WTerm : Term {
    DataPtr common, special;
    WTerm(DataPtr c, DataPtr s) : common(std::move(c)), special(std::move(s)) {}
    void apply(Builder& b) const override {
        const unsigned n = b.number_of_sites();
        if (n == 1) {
            b.connect(0, kStart, kEnd, special);
            return;
        }
        const unsigned s1 = b.allocate_signal(), s2 = b.allocate_signal(), last = n - 1;
        b.connect(0, kStart, s1, common);
        b.connect(0, kStart, s2, special);
        b.connect(last, s1, kEnd, special);
        b.connect(last, s2, kEnd, common);
        for (unsigned i = 1; i < last; ++i) {
            b.connect(i, s1, s1, common);
            b.connect(i, s1, s2, special);
            b.connect(i, s2, s2, common);
        }
    }
    void multiply_by(cd c) override { special = scaled(special, c); }
    Term* copy() const override { return new WTerm(*this); }
};

}  // namespace

struct NutcrackerMatrix {
    DataPtr m;
};
struct NutcrackerVector {
    DataPtr v;
};
struct NutcrackerOperator {
    std::vector<SitePtr> sites;
};
struct NutcrackerState {
    std::vector<SitePtr> sites;   // (br, bl, d); first unnormalised, the rest right-normalised
};
struct NutcrackerOperatorBuilder {
    Builder b;
};
struct NutcrackerStateBuilder {
    Builder b;
};
struct NutcrackerOperatorTerm {
    std::unique_ptr<Term> t;
};
struct NutcrackerStateTerm {
    std::unique_ptr<Term> t;
};
struct NutcrackerSerialization {
    std::string bytes;
};

namespace {

const cd* as_cd(const NutcrackerComplex* p) { return reinterpret_cast<const cd*>(p); }

template <typename T>
const T& need(const T* p, const char* what) {
    if (!p) throw std::invalid_argument(std::string("null ") + what);
    return *p;
}

// ---- protobuf wire format (nutcracker.proto) --------------------------------
void put_varint(std::string& o, uint64_t v) {
    while (v >= 0x80) {
        o.push_back((char)(v | 0x80));
        v >>= 7;
    }
    o.push_back((char)v);
}
void put_tag(std::string& o, unsigned field, unsigned wire) { put_varint(o, ((uint64_t)field << 3) | wire); }
void put_uint(std::string& o, unsigned field, uint64_t v) {
    put_tag(o, field, 0);
    put_varint(o, v);
}
void put_bytes(std::string& o, unsigned field, const std::string& b) {
    put_tag(o, field, 2);
    put_varint(o, b.size());
    o += b;
}
void put_packed_doubles(std::string& o, unsigned field, const std::vector<nc_complex>& z) {
    if (z.empty()) return;
    std::string b;
    b.resize(z.size() * 16);
    std::memcpy(&b[0], z.data(), b.size());   // little-endian IEEE doubles, real then imaginary
    put_bytes(o, field, b);
}
void put_packed_uints(std::string& o, unsigned field, const std::vector<uint32_t>& v) {
    if (v.empty()) return;
    std::string b;
    for (uint32_t x : v) put_varint(b, x);
    put_bytes(o, field, b);
}

struct Reader {
    const unsigned char* p;
    const unsigned char* end;
    bool done() const { return p >= end; }
    uint64_t varint() {
        uint64_t v = 0;
        for (int shift = 0; shift < 64; shift += 7) {
            if (p >= end) throw std::runtime_error("truncated protobuf message");
            const unsigned char c = *p++;
            v |= (uint64_t)(c & 0x7f) << shift;
            if (!(c & 0x80)) return v;
        }
        throw std::runtime_error("malformed protobuf varint");
    }
    Reader sub() {
        const uint64_t n = varint();
        if ((uint64_t)(end - p) < n) throw std::runtime_error("truncated protobuf message");
        Reader r{p, p + n};
        p += n;
        return r;
    }
    void skip(unsigned wire) {
        if (wire == 0) varint();
        else if (wire == 1) advance(8);
        else if (wire == 2) sub();
        else if (wire == 5) advance(4);
        else throw std::runtime_error("unsupported protobuf wire type " + std::to_string(wire));
    }
    void advance(size_t n) {
        if ((size_t)(end - p) < n) throw std::runtime_error("truncated protobuf message");
        p += n;
    }
};

std::vector<double> read_doubles(Reader& r, unsigned wire) {
    std::vector<double> out;
    if (wire == 2) {
        Reader s = r.sub();
        if ((s.end - s.p) % 8) throw std::runtime_error("malformed packed double field");
        out.resize((s.end - s.p) / 8);
        std::memcpy(out.data(), s.p, out.size() * 8);
    } else if (wire == 1) {
        double d;
        if (r.end - r.p < 8) throw std::runtime_error("truncated protobuf message");
        std::memcpy(&d, r.p, 8);
        r.p += 8;
        out.push_back(d);
    } else {
        throw std::runtime_error("wrong wire type for a double field");
    }
    return out;
}
std::vector<uint32_t> read_uints(Reader& r, unsigned wire) {
    std::vector<uint32_t> out;
    if (wire == 2) {
        Reader s = r.sub();
        while (!s.done()) out.push_back((uint32_t)s.varint());
    } else if (wire == 0) {
        out.push_back((uint32_t)r.varint());
    } else {
        throw std::runtime_error("wrong wire type for an integer field");
    }
    return out;
}

// Unique sites (shared pointers, then equal content) and the 0-based sequence
// (deconstructOperatorTo).
void deconstruct(const std::vector<SitePtr>& sites, std::vector<SitePtr>& unique, std::vector<uint32_t>& seq) {
    for (const SitePtr& s : sites) {
        size_t k = 0;
        for (; k < unique.size(); ++k) {
            const SiteData &a = *unique[k], &b = *s;
            if (unique[k] == s || (a.d == b.d && a.cl == b.cl && a.cr == b.cr && a.idx == b.idx &&
                                   a.W.size() == b.W.size() &&
                                   std::memcmp(a.W.data(), b.W.data(), a.W.size() * sizeof(nc_complex)) == 0))
                break;
        }
        if (k == unique.size()) unique.push_back(s);
        seq.push_back((uint32_t)k);
    }
}

// constructOperatorFrom (io.hpp:350-370), 0-based sequence.
std::vector<SitePtr> construct_operator(const std::vector<SitePtr>& unique, const std::vector<uint32_t>& seq) {
    if (seq.empty()) throw std::runtime_error("No operator sites were specified.");
    std::vector<SitePtr> out;
    for (uint32_t index : seq) {
        if (index >= unique.size())
            throw std::runtime_error("When reading in an operator, a reference to the non-existent operator site "
                                     "number " + std::to_string(index) + " appeared in the sequence.");
        const SitePtr& s = unique[index];
        if (out.empty()) {
            if (s->cl != 1)
                throw std::runtime_error("The left dimension of the left-most site must be one but instead is " +
                                         std::to_string(s->cl) + ".");
        } else if (s->cl != out.back()->cr) {
            const size_t n = out.size();
            throw std::runtime_error("The left dimension (" + std::to_string(s->cl) + ") of site " + std::to_string(n - 1) +
                                     " does not match the right dimension (" + std::to_string(out.back()->cr) +
                                     ") of site " + std::to_string(n) + ".  (" + std::to_string(s->cl) +
                                     " != " + std::to_string(out.back()->cr) + ")");
        }
        out.push_back(s);
    }
    if (out.back()->cr != 1)
        throw std::runtime_error("The right dimension of the right-most site must be one but instead is " +
                                 std::to_string(out.back()->cr) + ".");
    return out;
}

// OperatorBuffer (nutcracker.proto; protobuf.cpp:41-99): unique sites and the 0-based sequence.
void parse_operator_buffer(const void* buffer, size_t size, std::vector<SitePtr>& unique, std::vector<uint32_t>& seq) {
    if (!buffer && size) throw std::invalid_argument("null buffer");
    const unsigned char* b = static_cast<const unsigned char*>(buffer);
    Reader r{b, b + size};
    while (!r.done()) {
        const uint64_t tag = r.varint();
        const unsigned field = (unsigned)(tag >> 3), wire = (unsigned)(tag & 7);
        if (field == 1 && wire == 2) {
            Reader m = r.sub();
            auto s = std::make_shared<SiteData>();
            uint64_t nnz = 0;
            std::vector<double> data;
            while (!m.done()) {
                const uint64_t t = m.varint();
                const unsigned f = (unsigned)(t >> 3), w = (unsigned)(t & 7);
                if (f >= 1 && f <= 4 && w == 0) {
                    const uint64_t v = m.varint();
                    if (f == 1) nnz = v;
                    else if (f == 2) s->d = (uint32_t)v;
                    else if (f == 3) s->cl = (uint32_t)v;
                    else s->cr = (uint32_t)v;
                } else if (f == 5) {
                    std::vector<double> d = read_doubles(m, w);
                    data.insert(data.end(), d.begin(), d.end());
                } else if (f == 6) {
                    std::vector<uint32_t> i = read_uints(m, w);
                    s->idx.insert(s->idx.end(), i.begin(), i.end());
                } else {
                    m.skip(w);
                }
            }
            if (data.size() != 2 * nnz * s->d * s->d || s->idx.size() != 2 * nnz)
                throw std::runtime_error("operator site buffer sizes do not match its number of matrices");
            for (uint32_t k = 0; k < 2 * nnz; ++k) {
                const uint32_t lim = (k % 2 == 0) ? s->cl : s->cr;
                if (s->idx[k] < 1 || s->idx[k] > lim) throw std::runtime_error("operator site index out of range");
            }
            s->W.resize(data.size() / 2);
            std::memcpy(s->W.data(), data.data(), data.size() * sizeof(double));
            unique.push_back(s);
        } else if (field == 2) {
            std::vector<uint32_t> v = read_uints(r, wire);
            seq.insert(seq.end(), v.begin(), v.end());
        } else {
            r.skip(wire);
        }
    }
}

std::vector<DataPtr> components_of(const NutcrackerMatrix* const* c, unsigned n) {
    std::vector<DataPtr> v;
    for (unsigned i = 0; i < n; ++i) v.push_back(need(c[i], "matrix").m);
    return v;
}
std::vector<DataPtr> components_of(const NutcrackerVector* const* c, unsigned n) {
    std::vector<DataPtr> v;
    for (unsigned i = 0; i < n; ++i) v.push_back(need(c[i], "vector").v);
    return v;
}

}  // namespace

extern "C" {

// ---- errors (errors.cpp) ----
void Nutcracker_clearError(void) { t_error.reset(); }
char const* Nutcracker_getError(void) { return t_error ? t_error->c_str() : nullptr; }
void Nutcracker_setError(char const* message) { set_error(message ? message : ""); }

// ---- matrices (matrix.cpp) ----
void Nutcracker_Matrix_free(NutcrackerMatrix* matrix) { delete matrix; }

static NutcrackerMatrix const* pauli(int which) {
    static const NutcrackerMatrix* p[4] = {nullptr, nullptr, nullptr, nullptr};
    static const bool init = [] {
        const cd I[4] = {1, 0, 0, 1}, X[4] = {0, 1, 1, 0}, Y[4] = {0, cd(0, -1), cd(0, 1), 0}, Z[4] = {1, 0, 0, -1};
        p[0] = new NutcrackerMatrix{make_matrix(2, I)};
        p[1] = new NutcrackerMatrix{make_matrix(2, X)};
        p[2] = new NutcrackerMatrix{make_matrix(2, Y)};
        p[3] = new NutcrackerMatrix{make_matrix(2, Z)};
        return true;
    }();
    (void)init;
    return p[which];
}
NutcrackerMatrix const* Nutcracker_Matrix_getPauliI(void) { return pauli(0); }
NutcrackerMatrix const* Nutcracker_Matrix_getPauliX(void) { return pauli(1); }
NutcrackerMatrix const* Nutcracker_Matrix_getPauliY(void) { return pauli(2); }
NutcrackerMatrix const* Nutcracker_Matrix_getPauliZ(void) { return pauli(3); }

// The exported constants of includes/nutcracker.h:29-35 (defined in the
// reference's c-interface/matrix.cpp:8-11): the same library-owned objects
// the getters return, set when the library is loaded.
NutcrackerMatrix const *Nutcracker_Matrix_Pauli_I = pauli(0), *Nutcracker_Matrix_Pauli_X = pauli(1),
                       *Nutcracker_Matrix_Pauli_Y = pauli(2), *Nutcracker_Matrix_Pauli_Z = pauli(3);

NutcrackerMatrix* Nutcracker_Matrix_new(uint32_t dimension, NutcrackerComplex const* data) {
    C_BEGIN
    if (!data && dimension) throw std::invalid_argument("null matrix data");
    return new NutcrackerMatrix{make_matrix(dimension, as_cd(data))};
    C_END(nullptr)
}
NutcrackerMatrix* Nutcracker_Matrix_newDiagonal(uint32_t dimension, NutcrackerComplex const* data) {
    C_BEGIN
    if (!data && dimension) throw std::invalid_argument("null matrix data");
    std::vector<cd> a((size_t)dimension * dimension, cd(0, 0));
    for (uint32_t i = 0; i < dimension; ++i) a[(size_t)i * dimension + i] = as_cd(data)[i];
    return new NutcrackerMatrix{make_matrix(dimension, a.data())};
    C_END(nullptr)
}
NutcrackerMatrix* Nutcracker_Matrix_add(NutcrackerMatrix const* x, NutcrackerMatrix const* y) {
    C_BEGIN
    return new NutcrackerMatrix{summed(need(x, "matrix").m, need(y, "matrix").m)};
    C_END(nullptr)
}
NutcrackerMatrix* Nutcracker_Matrix_multiply(NutcrackerComplex const* c, NutcrackerMatrix const* x) {
    C_BEGIN
    return new NutcrackerMatrix{scaled(need(x, "matrix").m, *as_cd(&need(c, "coefficient")))};
    C_END(nullptr)
}
uint32_t Nutcracker_Matrix_getSize(NutcrackerMatrix const* x) { return x ? x->m->n : 0; }
void Nutcracker_Matrix_getElementAtCoordinate(NutcrackerMatrix const* x, uint32_t i, uint32_t j,
                                              NutcrackerComplex* element) {
    C_BEGIN
    const Data& m = *need(x, "matrix").m;
    if (i >= m.n || j >= m.n) throw std::out_of_range("matrix coordinate out of range");
    *reinterpret_cast<cd*>(element) = m.a[(size_t)i * m.n + j];
    C_END()
}

// ---- vectors (vector.cpp) ----
void Nutcracker_Vector_free(NutcrackerVector* vector) { delete vector; }

// The qubit basis vectors up = (1, 0) and down = (0, 1) of
// includes/nutcracker.h:148-151 (c-interface/vector.cpp:10-11,
// utilities.cpp:120-121), owned by the library.
static NutcrackerVector const* qubit(int which) {
    static const NutcrackerVector* q[2] = {nullptr, nullptr};
    static const bool init = [] {
        const cd up[2] = {1, 0}, down[2] = {0, 1};
        q[0] = new NutcrackerVector{make_vector(2, up)};
        q[1] = new NutcrackerVector{make_vector(2, down)};
        return true;
    }();
    (void)init;
    return q[which];
}
NutcrackerVector const *Nutcracker_Vector_Qubit_Up = qubit(0), *Nutcracker_Vector_Qubit_Down = qubit(1);
NutcrackerVector* Nutcracker_Vector_new(uint32_t physical_dimension, NutcrackerComplex const* data) {
    C_BEGIN
    if (!data && physical_dimension) throw std::invalid_argument("null vector data");
    return new NutcrackerVector{make_vector(physical_dimension, as_cd(data))};
    C_END(nullptr)
}
NutcrackerVector* Nutcracker_Vector_newBasis(uint32_t physical_dimension, uint32_t observed_value) {
    C_BEGIN
    if (observed_value >= physical_dimension)
        throw std::out_of_range("observed value " + std::to_string(observed_value) + " out of range for dimension " +
                                std::to_string(physical_dimension));
    std::vector<cd> v(physical_dimension, cd(0, 0));
    v[observed_value] = 1;
    return new NutcrackerVector{make_vector(physical_dimension, v.data())};
    C_END(nullptr)
}
NutcrackerVector* Nutcracker_Vector_add(NutcrackerVector const* x, NutcrackerVector const* y) {
    C_BEGIN
    return new NutcrackerVector{summed(need(x, "vector").v, need(y, "vector").v)};
    C_END(nullptr)
}
NutcrackerVector* Nutcracker_Vector_multiply(NutcrackerComplex const* c, NutcrackerVector const* x) {
    C_BEGIN
    return new NutcrackerVector{scaled(need(x, "vector").v, *as_cd(&need(c, "coefficient")))};
    C_END(nullptr)
}
uint32_t Nutcracker_Vector_getSize(NutcrackerVector const* x) { return x ? x->v->n : 0; }
void Nutcracker_Vector_getElementAtIndex(NutcrackerVector const* x, uint32_t index, NutcrackerComplex* element) {
    C_BEGIN
    const Data& v = *need(x, "vector").v;
    if (index >= v.n) throw std::out_of_range("vector index out of range");
    *reinterpret_cast<cd*>(element) = v.a[index];
    C_END()
}

// ---- operator builder and terms ----
NutcrackerOperatorBuilder* Nutcracker_OperatorBuilder_new(uint32_t number_of_sites, uint32_t* dimensions) {
    C_BEGIN
    if (!dimensions && number_of_sites) throw std::invalid_argument("null dimensions");
    return new NutcrackerOperatorBuilder{Builder(std::vector<uint32_t>(dimensions, dimensions + number_of_sites), true)};
    C_END(nullptr)
}
NutcrackerOperatorBuilder* Nutcracker_OperatorBuilder_newSimple(uint32_t number_of_sites, uint32_t physical_dimension) {
    C_BEGIN
    return new NutcrackerOperatorBuilder{Builder(std::vector<uint32_t>(number_of_sites, physical_dimension), true)};
    C_END(nullptr)
}
void Nutcracker_OperatorBuilder_free(NutcrackerOperatorBuilder* builder) { delete builder; }
uint32_t Nutcracker_OperatorBuilder_numberOfSites(NutcrackerOperatorBuilder const* builder) {
    return builder ? builder->b.number_of_sites() : 0;
}
uint32_t Nutcracker_OperatorBuilder_dimensionOfSite(NutcrackerOperatorBuilder const* builder, uint32_t site_number) {
    C_BEGIN
    return need(builder, "builder").b.dimension_of_site(site_number);
    C_END(0)
}
void Nutcracker_OperatorBuilder_addProductTerm(NutcrackerOperatorBuilder* builder,
                                               NutcrackerMatrix const* const* components) {
    C_BEGIN
    Builder& b = const_cast<Builder&>(need(builder, "builder").b);
    b.add_product_term(components_of(components, b.number_of_sites()));
    C_END()
}
void Nutcracker_OperatorBuilder_addTerm(NutcrackerOperatorBuilder* builder, NutcrackerOperatorTerm* term) {
    C_BEGIN
    need(term, "term").t->apply(const_cast<Builder&>(need(builder, "builder").b));
    C_END()
}
NutcrackerOperator* Nutcracker_OperatorBuilder_compileCustomized(NutcrackerOperatorBuilder* builder, bool optimize,
                                                                 bool add_start_and_end_loops) {
    C_BEGIN
    Specification spec = need(builder, "builder").b.specification(add_start_and_end_loops);
    if (optimize) spec.optimize();
    return new NutcrackerOperator{spec.compile(operator_site)};
    C_END(nullptr)
}
NutcrackerOperator* Nutcracker_OperatorBuilder_compile(NutcrackerOperatorBuilder* builder) {
    return Nutcracker_OperatorBuilder_compileCustomized(builder, true, true);
}

void Nutcracker_OperatorTerm_free(NutcrackerOperatorTerm* term) { delete term; }
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_add(NutcrackerOperatorTerm const* x, NutcrackerOperatorTerm const* y) {
    C_BEGIN
    return new NutcrackerOperatorTerm{std::unique_ptr<Term>(new SumTerm(need(x, "term").t.get(), need(y, "term").t.get()))};
    C_END(nullptr)
}
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_multiply(NutcrackerComplex const* c, NutcrackerOperatorTerm const* x) {
    C_BEGIN
    std::unique_ptr<Term> t(need(x, "term").t->copy());
    t->multiply_by(*as_cd(&need(c, "coefficient")));
    return new NutcrackerOperatorTerm{std::move(t)};
    C_END(nullptr)
}
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_LocalExternalField(uint32_t site_number,
                                                                          NutcrackerMatrix const* field_matrix) {
    C_BEGIN
    return new NutcrackerOperatorTerm{
        std::unique_ptr<Term>(new LocalExternalField(site_number, need(field_matrix, "matrix").m))};
    C_END(nullptr)
}
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_GlobalExternalField(NutcrackerMatrix const* field_matrix) {
    C_BEGIN
    return new NutcrackerOperatorTerm{std::unique_ptr<Term>(new GlobalExternalField(need(field_matrix, "matrix").m))};
    C_END(nullptr)
}
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_LocalNeighborCouplingField(
    uint32_t site_number, NutcrackerMatrix const* left_field_matrix, NutcrackerMatrix const* right_field_matrix) {
    C_BEGIN
    return new NutcrackerOperatorTerm{std::unique_ptr<Term>(new LocalNeighborCouplingField(
        site_number, need(left_field_matrix, "matrix").m, need(right_field_matrix, "matrix").m))};
    C_END(nullptr)
}
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_GlobalNeighborCouplingField(
    NutcrackerMatrix const* left_field_matrix, NutcrackerMatrix const* right_field_matrix) {
    C_BEGIN
    return new NutcrackerOperatorTerm{std::unique_ptr<Term>(
        new GlobalNeighborCouplingField(need(left_field_matrix, "matrix").m, need(right_field_matrix, "matrix").m))};
    C_END(nullptr)
}
NutcrackerOperatorTerm* Nutcracker_OperatorTerm_create_TransverseIsingField(
    NutcrackerMatrix const* external_field_matrix, NutcrackerMatrix const* left_coupling_field_matrix,
    NutcrackerMatrix const* right_coupling_field_matrix) {
    C_BEGIN
    GlobalExternalField ext(need(external_field_matrix, "matrix").m);
    GlobalNeighborCouplingField nb(need(left_coupling_field_matrix, "matrix").m,
                                   need(right_coupling_field_matrix, "matrix").m);
    return new NutcrackerOperatorTerm{std::unique_ptr<Term>(new SumTerm(&ext, &nb))};
    C_END(nullptr)
}

void Nutcracker_Operator_free(NutcrackerOperator* op) { delete op; }

// OperatorBuffer (protobuf.cpp:25-99)
NutcrackerSerialization* Nutcracker_Operator_serialize(NutcrackerOperator const* op) {
    C_BEGIN
    std::vector<SitePtr> unique;
    std::vector<uint32_t> seq;
    deconstruct(need(op, "operator").sites, unique, seq);
    std::string out;
    for (const SitePtr& s : unique) {
        std::string m;
        put_uint(m, 1, s->idx.size() / 2);
        put_uint(m, 2, s->d);
        put_uint(m, 3, s->cl);
        put_uint(m, 4, s->cr);
        put_packed_doubles(m, 5, s->W);
        put_packed_uints(m, 6, s->idx);
        put_bytes(out, 1, m);
    }
    put_packed_uints(out, 2, seq);
    return new NutcrackerSerialization{out};
    C_END(nullptr)
}
NutcrackerOperator* Nutcracker_Operator_deserialize(uint32_t size, void const* buffer) {
    C_BEGIN
    std::vector<SitePtr> unique;
    std::vector<uint32_t> seq;
    parse_operator_buffer(buffer, size, unique, seq);
    return new NutcrackerOperator{construct_operator(unique, seq)};
    C_END(nullptr)
}

// The protobuf input format of the command-line program (protobuf.cpp:110-131).
nc_parsed_operator* nc_protobuf_read_operator(const void* data, size_t length) {
    NC_ABI_BEGIN
    std::vector<SitePtr> unique;
    std::vector<uint32_t> seq;
    try {
        parse_operator_buffer(data, length, unique, seq);
    } catch (const std::runtime_error& e) {
        throw nc::Error(nc::NC_ERR_ARG, e.what());
    }
    auto op = std::make_unique<nc_parsed_operator>();
    for (const SitePtr& u : unique) {
        nc_parsed_operator::Site t;
        t.d = u->d;
        t.cl = u->cl;
        t.cr = u->cr;
        t.idx = u->idx;
        t.W = u->W;
        op->unique.push_back(std::move(t));
    }
    op->sequence = seq;
    op->assemble();
    return op.release();
    NC_ABI_END
    return nullptr;
}

// ---- serialization (serialization.cpp) ----
void Nutcracker_Serialization_free(NutcrackerSerialization* s) { delete s; }
uint32_t Nutcracker_Serialization_getSize(NutcrackerSerialization* s) { return s ? (uint32_t)s->bytes.size() : 0; }
void Nutcracker_Serialization_write(NutcrackerSerialization* s, void* buffer) {
    if (s && buffer && !s->bytes.empty()) std::memcpy(buffer, s->bytes.data(), s->bytes.size());
}

// ---- version (version.cpp) ----
static const uint32_t kVersion[3] = {1, 0, 0};
uint32_t Nutcracker_Version_getComponent(uint32_t index) { return index < 3 ? kVersion[index] : 0; }
uint32_t Nutcracker_Version_getSize(void) { return 3; }
char const* Nutcracker_Version_getString(void) { return "1.0.0"; }
void Nutcracker_Version_write(uint32_t* version) {
    if (version) std::memcpy(version, kVersion, sizeof kVersion);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// States and solves: GPU work through the library's chain and Level-0 entry
// points (each stages its host buffers through the calling thread's stream).
// ---------------------------------------------------------------------------
namespace {

[[noreturn]] void library_error() {
    throw std::runtime_error(nc_last_error() ? nc_last_error() : "library error");
}

// State(CopyFrom<sites>) (states.hpp:473-488): the last site scaled to unit
// norm, then the orthogonality centre moved to the first site, each site
// passed becoming right-normalised (norm_denorm_going_left_) and each new
// centre renormalised (states.cpp:94-164), so the state has unit norm.
std::vector<SitePtr> canonical_state(const std::vector<SitePtr>& sites) {
    if (sites.empty()) throw std::runtime_error("a state needs at least one site");
    SiteData current = *sites.back();
    double nrm = 0;
    for (const nc_complex& z : current.W) nrm += z.re * z.re + z.im * z.im;
    nrm = std::sqrt(nrm);
    if (nrm == 0) throw std::runtime_error("cannot normalise a zero state site");
    for (nc_complex& z : current.W) {
        z.re /= nrm;
        z.im /= nrm;
    }
    std::vector<SitePtr> rest;
    for (size_t k = sites.size() - 1; k-- > 0;) {
        const SiteData& A = *sites[k];   // (bm, bl, dl) with bm = A.cr
        if (A.cr != current.cl) throw std::runtime_error("state site dimensions do not match");
        SiteData denA = A, normB = current;
        const uint32_t bl = A.cl, bm = A.cr, br = current.cr, dl = A.d, dr = current.d;
        if (norm_denorm_going_left_(&bl, &bm, &br, &dl, &dr, A.W.data(), current.W.data(), denA.W.data(),
                                    normB.W.data()) != 0)
            library_error();
        rest.push_back(std::make_shared<SiteData>(normB));
        // the new centre is renormalised, as the reference's cursor moves do
        double n2 = 0;
        for (const nc_complex& z : denA.W) n2 += z.re * z.re + z.im * z.im;
        const double inv = n2 > 0 ? 1.0 / std::sqrt(n2) : 1.0;
        for (nc_complex& z : denA.W) {
            z.re *= inv;
            z.im *= inv;
        }
        current = denA;
    }
    std::vector<SitePtr> out{std::make_shared<SiteData>(current)};
    for (size_t k = rest.size(); k-- > 0;) out.push_back(rest[k]);
    return out;
}

cd overlap(const std::vector<SitePtr>& s1, const std::vector<SitePtr>& s2) {
    if (s1.size() != s2.size()) throw std::runtime_error("the states have different numbers of sites");
    std::vector<nc_complex> env{nc_complex{1, 0}};
    for (size_t k = 0; k < s1.size(); ++k) {
        const SiteData &a = *s1[k], &b = *s2[k];
        if (a.d != b.d) throw std::runtime_error("the states have different physical dimensions");
        std::vector<nc_complex> ov(a.W.size()), next((size_t)b.cr * a.cr);
        form_overlap_site_tensor_(&a.cr, &a.cl, &a.d, a.W.data(), ov.data());
        if (nc_last_status() != 0) library_error();
        contract_vs_left_(&a.cl, &a.cr, &b.cl, &b.cr, &a.d, env.data(), ov.data(), b.W.data(), next.data());
        if (nc_last_status() != 0) library_error();
        env.swap(next);
    }
    return cd(env[0].re, env[0].im);
}

cd expectation(const std::vector<SitePtr>& state, const std::vector<SitePtr>& op) {
    if (state.size() != op.size()) throw std::runtime_error("the state and the operator have different numbers of sites");
    std::vector<nc_complex> env{nc_complex{1, 0}};
    for (size_t k = 0; k < state.size(); ++k) {
        const SiteData &s = *state[k], &o = *op[k];
        if (s.d != o.d) throw std::runtime_error("the state and the operator have different physical dimensions");
        const uint32_t nnz = (uint32_t)(o.idx.size() / 2);
        std::vector<nc_complex> next((size_t)s.cr * s.cr * o.cr);
        contract_sos_left_(&s.cl, &s.cr, &o.cl, &o.cr, &s.d, env.data(), &nnz, o.idx.data(), o.W.data(), s.W.data(),
                           next.data());
        if (nc_last_status() != 0) library_error();
        env.swap(next);
    }
    return cd(env[0].re, env[0].im);
}

std::vector<nc_operator_site> site_structs(const std::vector<SitePtr>& op) {
    std::vector<nc_operator_site> v;
    for (const SitePtr& s : op)
        v.push_back(nc_operator_site{s->d, s->cl, s->cr, (uint32_t)(s->idx.size() / 2), s->idx.data(), s->W.data()});
    return v;
}

// Nutcracker_Operator_simpleSolve* (operator.cpp:20-56): least values, initial
// bond dimension 2, sanity 1e-12, site 1e-9, sweep and chain 1e-8; the chain's
// state per level in the reference's canonical form (centre on site 0).
void simple_solve(const NutcrackerOperator& op, uint32_t levels, float* eigenvalues, NutcrackerState** vectors) {
    nc_chain_options o;
    nc_chain_options_init(&o);
    std::snprintf(o.optimizer_mode, sizeof o.optimizer_mode, "<v");
    o.initial_bandwidth_dimension = 2;
    o.sanity_check_threshold = 1e-12;
    o.site_convergence_threshold = 1e-9;
    o.sweep_convergence_threshold = 1e-8;
    o.chain_convergence_threshold = 1e-8;
    std::vector<nc_operator_site> sites = site_structs(op.sites);
    nc_chain* ch = nc_chain_create((uint32_t)sites.size(), sites.data(), &o);
    if (!ch) library_error();
    std::unique_ptr<nc_chain, void (*)(nc_chain*)> guard(ch, nc_chain_free);
    for (uint32_t k = 0; k < levels; ++k) {
        if (k > 0 && (nc_chain_construct_and_add_projector_from_state(ch) != 0 || nc_chain_reset(ch) != 0))
            library_error();
        double e = 0;
        if (nc_chain_optimize_chain(ch) != 0 || nc_chain_get_energy(ch, &e) != 0) library_error();
        if (eigenvalues) eigenvalues[k] = (float)e;
        if (vectors) {
            if (nc_chain_move_to(ch, 0) != 0) library_error();
            auto st = new NutcrackerState;
            for (uint32_t i = 0; i < sites.size(); ++i) {
                uint32_t dims[3];
                if (nc_chain_get_site(ch, i, nullptr, dims) != 0) library_error();
                auto s = std::make_shared<SiteData>();
                s->cr = dims[0];
                s->cl = dims[1];
                s->d = dims[2];
                s->W.resize((size_t)dims[0] * dims[1] * dims[2]);
                if (nc_chain_get_site(ch, i, s->W.data(), dims) != 0) {
                    delete st;
                    library_error();
                }
                st->sites.push_back(s);
            }
            vectors[k] = st;
        }
    }
}

}  // namespace

extern "C" {

void Nutcracker_Operator_simpleSolveForLeastEigenvalues(NutcrackerOperator const* op, uint32_t number_of_levels,
                                                        float* eigenvalues) {
    C_BEGIN
    simple_solve(need(op, "operator"), number_of_levels, eigenvalues, nullptr);
    C_END()
}
void Nutcracker_Operator_simpleSolveForLeastEigenvaluesWithEigenvectors(NutcrackerOperator const* op,
                                                                        uint32_t number_of_levels,
                                                                        float* eigenvalues,
                                                                        NutcrackerState** eigenvectors) {
    C_BEGIN
    simple_solve(need(op, "operator"), number_of_levels, eigenvalues, eigenvectors);
    C_END()
}

void Nutcracker_State_free(NutcrackerState* state) { delete state; }
void Nutcracker_State_computeOverlap(NutcrackerState const* state1, NutcrackerState const* state2,
                                     NutcrackerComplex* result) {
    C_BEGIN
    *reinterpret_cast<cd*>(result) = overlap(need(state1, "state").sites, need(state2, "state").sites);
    C_END()
}
void Nutcracker_State_computeExpectation(NutcrackerState const* state, NutcrackerOperator const* op,
                                         NutcrackerComplex* result) {
    C_BEGIN
    *reinterpret_cast<cd*>(result) = expectation(need(state, "state").sites, need(op, "operator").sites);
    C_END()
}

// StateBuffer (protobuf.hpp:87-93, protobuf.cpp:101-120): the first site with
// normalization MIDDLE, the others RIGHT.
NutcrackerSerialization* Nutcracker_State_serialize(NutcrackerState const* state) {
    C_BEGIN
    std::string out;
    const std::vector<SitePtr>& sites = need(state, "state").sites;
    for (size_t k = 0; k < sites.size(); ++k) {
        const SiteData& s = *sites[k];
        std::string m;
        put_uint(m, 1, k == 0 ? 0 : 2);
        put_uint(m, 2, s.d);
        put_uint(m, 3, s.cl);
        put_uint(m, 4, s.cr);
        put_packed_doubles(m, 5, s.W);
        put_bytes(out, 1, m);
    }
    return new NutcrackerSerialization{out};
    C_END(nullptr)
}
NutcrackerState* Nutcracker_State_deserialize(uint32_t size, void const* buffer) {
    C_BEGIN
    if (!buffer && size) throw std::invalid_argument("null buffer");
    const unsigned char* b = static_cast<const unsigned char*>(buffer);
    Reader r{b, b + size};
    auto st = std::unique_ptr<NutcrackerState>(new NutcrackerState);
    while (!r.done()) {
        const uint64_t tag = r.varint();
        const unsigned field = (unsigned)(tag >> 3), wire = (unsigned)(tag & 7);
        if (field != 1 || wire != 2) {
            r.skip(wire);
            continue;
        }
        Reader m = r.sub();
        auto s = std::make_shared<SiteData>();
        std::vector<double> data;
        while (!m.done()) {
            const uint64_t t = m.varint();
            const unsigned f = (unsigned)(t >> 3), w = (unsigned)(t & 7);
            if (f >= 1 && f <= 4 && w == 0) {
                const uint64_t v = m.varint();
                if (f == 2) s->d = (uint32_t)v;
                else if (f == 3) s->cl = (uint32_t)v;
                else if (f == 4) s->cr = (uint32_t)v;
            } else if (f == 5) {
                std::vector<double> d = read_doubles(m, w);
                data.insert(data.end(), d.begin(), d.end());
            } else {
                m.skip(w);
            }
        }
        if (data.size() != 2ull * s->d * s->cl * s->cr)
            throw std::runtime_error("state site buffer size does not match its dimensions");
        s->W.resize(data.size() / 2);
        std::memcpy(s->W.data(), data.data(), data.size() * sizeof(double));
        if (!st->sites.empty() && st->sites.back()->cr != s->cl)
            throw std::runtime_error("state site dimensions do not match");
        st->sites.push_back(s);
    }
    if (st->sites.empty()) throw std::runtime_error("a state needs at least one site");
    return st.release();
    C_END(nullptr)
}

NutcrackerStateBuilder* Nutcracker_StateBuilder_new(uint32_t number_of_sites, uint32_t* dimensions) {
    C_BEGIN
    if (!dimensions && number_of_sites) throw std::invalid_argument("null dimensions");
    return new NutcrackerStateBuilder{Builder(std::vector<uint32_t>(dimensions, dimensions + number_of_sites), false)};
    C_END(nullptr)
}
NutcrackerStateBuilder* Nutcracker_StateBuilder_newSimple(uint32_t number_of_sites, uint32_t physical_dimension) {
    C_BEGIN
    return new NutcrackerStateBuilder{Builder(std::vector<uint32_t>(number_of_sites, physical_dimension), false)};
    C_END(nullptr)
}
void Nutcracker_StateBuilder_free(NutcrackerStateBuilder* builder) { delete builder; }
uint32_t Nutcracker_StateBuilder_numberOfSites(NutcrackerStateBuilder const* builder) {
    return builder ? builder->b.number_of_sites() : 0;
}
uint32_t Nutcracker_StateBuilder_dimensionOfSite(NutcrackerStateBuilder const* builder, uint32_t site_number) {
    C_BEGIN
    return need(builder, "builder").b.dimension_of_site(site_number);
    C_END(0)
}
void Nutcracker_StateBuilder_addProductTerm(NutcrackerStateBuilder* builder, NutcrackerVector const* const* components) {
    C_BEGIN
    Builder& b = const_cast<Builder&>(need(builder, "builder").b);
    b.add_product_term(components_of(components, b.number_of_sites()));
    C_END()
}
void Nutcracker_StateBuilder_addTerm(NutcrackerStateBuilder* builder, NutcrackerStateTerm* term) {
    C_BEGIN
    need(term, "term").t->apply(const_cast<Builder&>(need(builder, "builder").b));
    C_END()
}
NutcrackerState* Nutcracker_StateBuilder_compileCustomized(NutcrackerStateBuilder* builder, bool optimize) {
    C_BEGIN
    Specification spec = need(builder, "builder").b.specification(false);
    if (optimize) spec.optimize();
    return new NutcrackerState{canonical_state(spec.compile(state_site))};
    C_END(nullptr)
}
NutcrackerState* Nutcracker_StateBuilder_compile(NutcrackerStateBuilder* builder) {
    return Nutcracker_StateBuilder_compileCustomized(builder, true);
}

void Nutcracker_StateTerm_free(NutcrackerStateTerm* term) { delete term; }
NutcrackerStateTerm* Nutcracker_StateTerm_add(NutcrackerStateTerm const* x, NutcrackerStateTerm const* y) {
    C_BEGIN
    return new NutcrackerStateTerm{std::unique_ptr<Term>(new SumTerm(need(x, "term").t.get(), need(y, "term").t.get()))};
    C_END(nullptr)
}
NutcrackerStateTerm* Nutcracker_StateTerm_multiply(NutcrackerComplex const* c, NutcrackerStateTerm const* x) {
    C_BEGIN
    std::unique_ptr<Term> t(need(x, "term").t->copy());
    t->multiply_by(*as_cd(&need(c, "coefficient")));
    return new NutcrackerStateTerm{std::move(t)};
    C_END(nullptr)
}
NutcrackerStateTerm* Nutcracker_StateTerm_create_ProductWithOneSiteDifferent(uint32_t site_number,
                                                                             NutcrackerVector const* common_observation,
                                                                             NutcrackerVector const* special_observation) {
    C_BEGIN
    return new NutcrackerStateTerm{std::unique_ptr<Term>(new ProductWithOneSiteDifferent(
        site_number, need(common_observation, "vector").v, need(special_observation, "vector").v))};
    C_END(nullptr)
}
NutcrackerStateTerm* Nutcracker_StateTerm_create_W(NutcrackerVector const* common_observation,
                                                   NutcrackerVector const* special_observation, bool normalized) {
    C_BEGIN
    (void)normalized;
    return new NutcrackerStateTerm{std::unique_ptr<Term>(
        new WTerm(need(common_observation, "vector").v, need(special_observation, "vector").v))};
    C_END(nullptr)
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Checkpoint and resume of a chain's state in the StateBuffer layout
// (nutcracker.proto; the state the reference's protobuf outputter writes,
// protobuf.cpp:101-104): the centre moved to site 0, then every site.
// ---------------------------------------------------------------------------
extern "C" {

size_t nc_chain_serialize_state(nc_chain* chain, void* out, size_t capacity) {
    NC_ABI_BEGIN
    NC_ARG(chain != nullptr, "null chain");
    nc_chain_info info;
    if (nc_chain_get_info(chain, &info) != 0 || nc_chain_move_to(chain, 0) != 0)
        throw nc::Error(nc_last_status(), nc_last_error());
    std::string buf;
    for (uint32_t i = 0; i < info.number_of_sites; ++i) {
        uint32_t dims[3];
        if (nc_chain_get_site(chain, i, nullptr, dims) != 0) throw nc::Error(nc_last_status(), nc_last_error());
        std::vector<nc_complex> w((size_t)dims[0] * dims[1] * dims[2]);
        if (nc_chain_get_site(chain, i, w.data(), dims) != 0) throw nc::Error(nc_last_status(), nc_last_error());
        std::string m;
        put_uint(m, 1, i == 0 ? 0 : 2);
        put_uint(m, 2, dims[2]);
        put_uint(m, 3, dims[1]);
        put_uint(m, 4, dims[0]);
        put_packed_doubles(m, 5, w);
        put_bytes(buf, 1, m);
    }
    if (out && capacity >= buf.size()) std::memcpy(out, buf.data(), buf.size());
    return buf.size();
    NC_ABI_END
    return 0;
}

int nc_chain_deserialize_state(nc_chain* chain, const void* data, size_t length) {
    NC_ABI_BEGIN
    NC_ARG(chain != nullptr, "null chain");
    std::unique_ptr<NutcrackerState> st(Nutcracker_State_deserialize((uint32_t)length, data));
    if (!st) throw nc::Error(nc::NC_ERR_ARG, Nutcracker_getError() ? Nutcracker_getError() : "bad state buffer");
    std::vector<uint32_t> bonds{1};
    std::vector<const nc_complex*> sites;
    for (const SitePtr& s : st->sites) {
        NC_ARG(s->cl == bonds.back(), "state site dimensions do not match");
        bonds.push_back(s->cr);
        sites.push_back(s->W.data());
    }
    nc_chain_info info;
    if (nc_chain_get_info(chain, &info) != 0) throw nc::Error(nc_last_status(), nc_last_error());
    NC_ARG(sites.size() == info.number_of_sites, "the state has a different number of sites than the chain");
    for (uint32_t i = 0; i < info.number_of_sites; ++i) {
        uint32_t dims[3];
        if (nc_chain_get_site(chain, i, nullptr, dims) != 0) throw nc::Error(nc_last_status(), nc_last_error());
        NC_ARG(dims[2] == st->sites[i]->d, "the state's physical dimensions differ from the chain's");
    }
    if (nc_chain_set_state(chain, bonds.data(), sites.data()) != 0) throw nc::Error(nc_last_status(), nc_last_error());
    NC_ABI_END
    return nc::g_status;
}

}  // extern "C"
