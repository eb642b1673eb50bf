// Minimal stand-ins for the Rcpp types used by the reference's parsimony
// functions, so that those functions compile as plain C++ for the oracle
// pin (test infrastructure, see oracle/Makefile target ref).  Matrices are
// column-major like R's; only the members those functions use exist.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

// R's transient allocator and printf (the test process frees at exit)
inline char* R_alloc(size_t n, int size) { return static_cast<char*>(std::calloc(n ? n : 1, (size_t)size)); }
#define Rprintf std::printf

namespace Rcpp {

struct IntegerVector {
    std::vector<int> v;
    IntegerVector(int n = 0) : v((size_t)n, 0) {}
    int& operator()(int i) { return v[(size_t)i]; }
    int operator()(int i) const { return v[(size_t)i]; }
    int& operator[](int i) { return v[(size_t)i]; }
    int size() const { return (int)v.size(); }
    void fill(int x) { for (auto& e : v) e = x; }
};

struct LogicalVector {
    std::vector<int> v;
    LogicalVector(int n = 0) : v((size_t)n, 0) {}
    int& operator()(int i) { return v[(size_t)i]; }
    void fill(bool x) { for (auto& e : v) e = x ? 1 : 0; }
};

struct MatrixColumn {
    int* p;
    int n;
    operator IntegerVector() const {
        IntegerVector r(n);
        for (int i = 0; i < n; i++) r.v[(size_t)i] = p[i];
        return r;
    }
    MatrixColumn& operator=(const IntegerVector& x) {
        for (int i = 0; i < n; i++) p[i] = x.v[(size_t)i];
        return *this;
    }
};

struct IntegerMatrix {
    int nr = 0, nc = 0;
    std::vector<int> v;
    IntegerMatrix(int r = 0, int c = 0) : nr(r), nc(c), v((size_t)r * c, 0) {}
    int& operator()(int i, int j) { return v[(size_t)i + (size_t)j * nr]; }
    int nrow() const { return nr; }
    int ncol() const { return nc; }
    void fill(int x) { for (auto& e : v) e = x; }
    MatrixColumn column(int j) { return MatrixColumn{v.data() + (size_t)j * nr, nr}; }
};

template <class T>
struct NamedValue {
    std::string name;
    T value;
};

struct Named {
    std::string name;
    explicit Named(const char* n) : name(n) {}
    template <class T>
    NamedValue<T> operator=(const T& x) const { return NamedValue<T>{name, x}; }
};

// List::create keeps the matrices and vectors it is given, by name.
struct List {
    std::vector<std::pair<std::string, IntegerMatrix>> mats;
    std::vector<std::pair<std::string, IntegerVector>> vecs;
    void add(const NamedValue<IntegerMatrix>& x) { mats.emplace_back(x.name, x.value); }
    void add(const NamedValue<IntegerVector>& x) { vecs.emplace_back(x.name, x.value); }
    template <class... A>
    static List create(const A&... a) {
        List l;
        (l.add(a), ...);
        return l;
    }
};

}  // namespace Rcpp
