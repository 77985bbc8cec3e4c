// Harness around the reference's own C++ measures (query/cpp/spatial/traj.cpp:
// Traj::DTW :157-182, Traj::Frechet :129-154, Traj::ERP :185-239,
// Traj::HausdorffDistance :48-126).
//
// TEST INFRASTRUCTURE ONLY: this is the reference's CPU code path, used to pin
// the oracle and as the timed CPU baseline.  oracle/build.py compiles it
// together with the reference sources read in place (the embedded-CPython
// section of traj.cpp, TrajSimiGPU, is stripped at compile time) into
// oracle/_ref/libtsm_ref.so.  No reference source is copied into this repo.
//
// The reference has no EDR/LCSS in C++; tsm_ref_pairs returns -2 for them.
#include <atomic>
#include <cstdint>
#include <thread>
#include <vector>

#include "traj.h"

namespace {

struct RefSet {
    std::vector<Traj*> trajs;
};

Traj* make_traj(const float* pts, int64_t off, int32_t len, unsigned id) {
    Traj* t = new Traj();
    t->id = id;
    for (int32_t i = 0; i < len; ++i) {
        Point* p = new Point(pts[2 * (off + i)], pts[2 * (off + i) + 1]);
        if (i > 0) t->edges.push_back(new Edge(t->points.back(), p, id));
        t->points.push_back(p);
    }
    return t;
}

}  // namespace

extern "C" {

// Builds the reference Traj objects once (the reference builds them when it
// loads a dataset, outside any timed measure call).
void* tsm_ref_build(const float* pts, const int64_t* offs, const int32_t* lens, int64_t n_traj) {
    RefSet* s = new RefSet();
    s->trajs.reserve(n_traj);
    for (int64_t k = 0; k < n_traj; ++k) s->trajs.push_back(make_traj(pts, offs[k], lens[k], (unsigned)k));
    return s;
}

void tsm_ref_free(void* h) {
    RefSet* s = static_cast<RefSet*>(h);
    if (!s) return;
    for (Traj* t : s->trajs) delete t;
    delete s;
}

// measure: 0 DTW, 3 ERP, 4 discrete Frechet, 5 Hausdorff (same numbering as
// the CUDA library); 1 EDR and 2 LCSS have no reference C++ code (-2).
// One pair per task over nthreads worker threads, like the reference's
// multiprocessing.Pool over pairs.
int tsm_ref_pairs(void* h, int measure, const int32_t* idx_a, const int32_t* idx_b, int64_t n,
                  float gx, float gy, float* out, int nthreads) {
    RefSet* s = static_cast<RefSet*>(h);
    if (!s) return -1;
    if (measure == 1 || measure == 2) return -2;
    if (measure < 0 || measure > 5) return -1;
    if (nthreads < 1) nthreads = 1;
    std::atomic<int64_t> next(0);
    auto work = [&]() {
        Point g(gx, gy);
        for (;;) {
            int64_t k = next.fetch_add(1);
            if (k >= n) break;
            Traj* a = s->trajs[idx_a[k]];
            Traj* b = s->trajs[idx_b[k]];
            float r = 0.0f;
            switch (measure) {
                case 0: r = a->DTW(b); break;
                case 3: r = a->ERP(b, g); break;
                case 4: r = a->Frechet(b); break;
                case 5: r = a->HausdorffDistance(b); break;
            }
            out[k] = r;
        }
    };
    if (nthreads == 1) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t) pool.emplace_back(work);
        for (auto& th : pool) th.join();
    }
    return 0;
}

}  // extern "C"
