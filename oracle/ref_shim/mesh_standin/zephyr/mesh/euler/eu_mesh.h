// Stand-in for zephyr/mesh/euler/eu_mesh.h (TEST INFRASTRUCTURE ONLY).
//
// It provides the EuMesh / EuCell / EuFace / Children / Distributor surface
// that math/solver/sm_fluid.cpp, math/cfd/gradient.h and face_extra.h use,
// over plain arrays in the layout of AmrCells / AmrFaces (8 face slots per
// cell, UNDEFINED slots skipped in slot order; eu_prim.cpp:7-32,
// amr_faces.cpp:186-197).  The checker fills the geometry; the solver code
// that runs on it is the reference's own.
#pragma once

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>
#include <functional>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include <zephyr/geom/boundary.h>
#include <zephyr/geom/vector.h>
#include <zephyr/mesh/storage.h>
#include <zephyr/utils/mpi.h>
#include <zephyr/utils/threads.h>

namespace zephyr::mesh {

using geom::Boundary;
using geom::Vector3d;

struct ShimMesh {
    int n = 0;
    std::vector<Vector3d> center;
    std::vector<double> volume;
    std::vector<double> incircle;
    std::vector<int> flag;
    std::vector<int> boundary;  // 8 per cell
    std::vector<int> adj;       // 8 per cell
    std::vector<Vector3d> fnormal, fcenter;
    std::vector<double> farea;
    std::vector<std::vector<char>> fields;
    std::vector<size_t> elem;
};

class EuCell;

class EuFace {
public:
    EuFace(ShimMesh *m, int f) : m_(m), f_(f) {}
    const Vector3d &normal() const { return m_->fnormal[f_]; }
    const Vector3d &center() const { return m_->fcenter[f_]; }
    Boundary flag() const { return Boundary(m_->boundary[f_]); }
    bool is_boundary() const {  // amr_faces.h:157-161
        int b = m_->boundary[f_];
        return b != int(Boundary::INNER) && b != int(Boundary::PERIODIC) && b != int(Boundary::UNDEFINED);
    }
    double area() const { return m_->farea[f_]; }
    double area(bool axial) const { return m_->farea[f_]; }
    inline EuCell neib() const;
    template <typename T>
    const T &neib(Storable<T> s) const {
        return reinterpret_cast<const T *>(m_->fields[s.index].data())[m_->adj[f_]];
    }
    Vector3d neib_center() const { return m_->center[m_->adj[f_]]; }
    Vector3d symm_point(const Vector3d &p) const {  // amr_faces.h:197-199
        return p + 2.0 * (center() - p).dot(normal()) * normal();
    }
    int index() const { return f_; }
    void set_index(int f) { f_ = f; }

private:
    ShimMesh *m_;
    int f_;
};

class FaceIter {
public:
    FaceIter(ShimMesh *m, int f, int end) : face_(m, f), m_(m), end_(end) { skip(); }
    EuFace &operator*() { return face_; }
    FaceIter &operator++() {
        face_.set_index(face_.index() + 1);
        skip();
        return *this;
    }
    bool operator!=(const FaceIter &o) const { return face_.index() != o.face_.index(); }

private:
    void skip() {
        while (face_.index() < end_ && m_->boundary[face_.index()] == int(Boundary::UNDEFINED))
            face_.set_index(face_.index() + 1);
    }
    EuFace face_;
    ShimMesh *m_;
    int end_;
};

struct EuFaces {
    ShimMesh *m;
    int b, e;
    FaceIter begin() const { return FaceIter(m, b, e); }
    FaceIter end() const { return FaceIter(m, e, e); }
};

class EuCell {
public:
    EuCell(ShimMesh *m, int ic) : m_(m), ic_(ic) {}
    template <typename T>
    T &operator[](Storable<T> s) {
        return reinterpret_cast<T *>(m_->fields[s.index].data())[ic_];
    }
    template <typename T>
    const T &operator[](Storable<T> s) const {
        return reinterpret_cast<const T *>(m_->fields[s.index].data())[ic_];
    }
    const Vector3d &center() const { return m_->center[ic_]; }
    double volume() const { return m_->volume[ic_]; }
    double volume(bool axial) const { return m_->volume[ic_]; }
    EuFaces faces() const { return EuFaces{m_, 8 * ic_, 8 * ic_ + 8}; }
    double incircle_diameter() const { return m_->incircle[ic_]; }
    void set_flag(int f) { m_->flag[ic_] = f; }
    int flag() const { return m_->flag[ic_]; }
    int dim() const { return 2; }
    double linear_size() const { return std::sqrt(m_->volume[ic_]); }
    int index() const { return ic_; }

private:
    ShimMesh *m_;
    int ic_;
};

inline EuCell EuFace::neib() const { return EuCell(m_, m_->adj[f_]); }

class Children {
public:
    std::vector<EuCell> cells;
    auto begin() { return cells.begin(); }
    auto end() { return cells.end(); }
    auto begin() const { return cells.begin(); }
    auto end() const { return cells.end(); }
};

struct Distributor {
    using split_function = std::function<void(const EuCell &, Children &)>;
    using merge_function = std::function<void(const Children &, EuCell &)>;
    split_function split;
    merge_function merge;
};

class CellIter {
public:
    CellIter(ShimMesh *m, int ic) : m_(m), ic_(ic) {}
    EuCell operator*() const { return EuCell(m_, ic_); }
    CellIter &operator++() {
        ++ic_;
        return *this;
    }
    bool operator!=(const CellIter &o) const { return ic_ != o.ic_; }

private:
    ShimMesh *m_;
    int ic_;
};

class EuMesh {
public:
    explicit EuMesh(ShimMesh *m) : m_(m) {}
    template <typename T>
    Storable<T> add(const std::string &) {
        m_->fields.emplace_back(sizeof(T) * (size_t)m_->n, char(0));
        m_->elem.push_back(sizeof(T));
        return Storable<T>(int(m_->fields.size()) - 1);
    }
    // utils::threads::for_each (threads.h:64-90): the range is cut into
    // n_threads * 10 tasks run by n_threads workers; sequential below 2 threads.
    template <class F>
    void for_each(F &&f) {
        run_tasks([&](int b, int e) {
            for (int ic = b; ic < e; ++ic) {
                EuCell c(m_, ic);
                f(c);
            }
        });
    }
    // threads::min (threads.h:95-110): start from numeric_limits::max, std::min
    // per task, then over tasks (the minimum does not depend on the order).
    template <class F>
    double min(F &&f) {
        std::vector<double> part(std::max(1, n_threads) * 10 + 1, std::numeric_limits<double>::max());
        std::atomic<int> slot{0};
        run_tasks([&](int b, int e) {
            double r = std::numeric_limits<double>::max();
            for (int ic = b; ic < e; ++ic) r = std::min(r, f(EuCell(m_, ic)));
            part[slot.fetch_add(1)] = r;
        });
        double r = std::numeric_limits<double>::max();
        for (double x : part) r = std::min(r, x);
        return r;
    }
    void set_threads(int n) { n_threads = n; }

    template <class G>
    void run_tasks(G &&g) {
        int n = m_->n;
        if (n_threads < 2) {
            g(0, n);
            return;
        }
        int n_tasks = n_threads * 10;
        int chunk = (n + n_tasks - 1) / n_tasks;
        std::atomic<int> next{0};
        std::vector<std::thread> pool;
        for (int t = 0; t < n_threads; ++t)
            pool.emplace_back([&]() {
                for (;;) {
                    int k = next.fetch_add(1);
                    int b = k * chunk;
                    if (b >= n) break;
                    g(b, std::min(n, b + chunk));
                }
            });
        for (auto &th : pool) th.join();
    }
    template <class... Args>
    void sync(Args &&...) {}
    template <typename T>
    void swap(Storable<T> a, Storable<T> b) {
        std::swap(m_->fields[a.index], m_->fields[b.index]);
    }
    bool adaptive() const { return true; }
    CellIter begin() { return CellIter(m_, 0); }
    CellIter end() { return CellIter(m_, m_->n); }
    int n_cells() const { return m_->n; }
    ShimMesh *shim() { return m_; }

private:
    ShimMesh *m_;
    int n_threads = 1;
};

}  // namespace zephyr::mesh
