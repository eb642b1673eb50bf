// Minimal stand-ins for the Rcpp types used by the reference's CPU functions
// (src/functions.cpp), so that those functions compile as plain C++ for the
// oracle pin and the timed CPU baseline (test infrastructure, see the
// oracle/Makefile target ref).  Only the members those functions use exist.
//
// The copy rules follow Rcpp's: a vector or matrix is a handle, so copying
// one (passing it by value, assigning it) shares its storage; converting a
// matrix column to a vector makes a new vector; assigning a vector or another
// column to a matrix column copies the elements.  Matrices are column-major
// like R's.  Element access is unchecked (Rcpp's operator() on vectors checks
// bounds), so the functions run at least as fast here as under R.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <string>
#include <vector>

// R's transient allocator: memory lives until the wrapper that called the
// function releases it, as R releases it when the .Call returns.
inline std::vector<void*>& r_alloc_list() {
    thread_local std::vector<void*> l;
    return l;
}
inline char* R_alloc(size_t n, int size) {
    void* p = std::calloc(n ? n : 1, (size_t)size);
    r_alloc_list().push_back(p);
    return static_cast<char*>(p);
}
inline void r_alloc_release() {
    for (void* p : r_alloc_list()) std::free(p);
    r_alloc_list().clear();
}
#define Rprintf std::printf

// An R object handle; here only a pointer to a BigMatrix or a null result.
typedef void* SEXP;

// bigmemory's matrix and column accessor (column-major int storage).
struct BigMatrix {
    long nr = 0, nc = 0;
    int* d = nullptr;
    long nrow() const { return nr; }
    long ncol() const { return nc; }
};

template <class T>
struct MatrixAccessor {
    T* d;
    long nr;
    explicit MatrixAccessor(BigMatrix& m) : d(reinterpret_cast<T*>(m.d)), nr(m.nr) {}
    T* operator[](long j) const { return d + j * nr; }
};

namespace Rcpp {

template <class T>
struct XPtr {
    T* p;
    explicit XPtr(SEXP s) : p(static_cast<T*>(s)) {}
    T* operator->() const { return p; }
    T& operator*() const { return *p; }
};

template <class T>
struct Vec {
    std::shared_ptr<std::vector<T>> s;
    Vec(int n = 0) : s(std::make_shared<std::vector<T>>((size_t)n, T())) {}
    T& operator()(int i) const { return (*s)[(size_t)i]; }
    T& operator[](size_t i) const { return (*s)[i]; }
    int size() const { return (int)s->size(); }
    void fill(T x) const { for (auto& e : *s) e = x; }
    T* data() const { return s->data(); }
};

struct IntegerVector : Vec<int> {
    using Vec<int>::Vec;
};

struct NumericVector : Vec<double> {
    using Vec<double>::Vec;
};

struct LogicalVector : Vec<int> {
    using Vec<int>::Vec;
    void fill(bool x) const { Vec<int>::fill(x ? 1 : 0); }
};

struct MatrixColumn {
    int* p;
    int n;
    operator IntegerVector() const {
        IntegerVector r(n);
        for (int i = 0; i < n; i++) r[(size_t)i] = p[i];
        return r;
    }
    MatrixColumn& operator=(const IntegerVector& x) {
        for (int i = 0; i < n; i++) p[i] = x[(size_t)i];
        return *this;
    }
    MatrixColumn& operator=(const MatrixColumn& x) {
        if (p != x.p)
            for (int i = 0; i < n; i++) p[i] = x.p[i];
        return *this;
    }
    MatrixColumn(int* p_, int n_) : p(p_), n(n_) {}
    MatrixColumn(const MatrixColumn&) = default;
};

template <class T>
struct Mat {
    int nr = 0, nc = 0;
    std::shared_ptr<std::vector<T>> s;
    Mat(int r = 0, int c = 0) : nr(r), nc(c), s(std::make_shared<std::vector<T>>((size_t)r * c, T())) {}
    T& operator()(int i, int j) const { return (*s)[(size_t)i + (size_t)j * nr]; }
    int nrow() const { return nr; }
    int ncol() const { return nc; }
    void fill(T x) const { for (auto& e : *s) e = x; }
    T* data() const { return s->data(); }
};

struct IntegerMatrix : Mat<int> {
    using Mat<int>::Mat;
    MatrixColumn column(int j) const { return MatrixColumn(s->data() + (size_t)j * nr, nr); }
};

struct NumericMatrix : Mat<double> {
    using Mat<double>::Mat;
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

// List::create keeps the matrices and vectors it is given, by name; a List
// made from a null SEXP (a function's `return 0;`) is marked null.
struct List {
    std::vector<std::pair<std::string, IntegerMatrix>> mats;
    std::vector<std::pair<std::string, IntegerVector>> vecs;
    bool null = false;
    List() = default;
    List(SEXP s) : null(s == nullptr) {}
    IntegerVector operator[](const char* name) const {
        for (auto& x : vecs)
            if (x.first == name) return x.second;
        return IntegerVector(0);
    }
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
