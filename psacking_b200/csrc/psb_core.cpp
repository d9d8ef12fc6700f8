// psb_core.cpp — pybind11 module `psacking_b200._core`.
//
// Same names, arguments, return tuples and error behaviour as the reference's
// module `spectral_packer._core` (spectral_packing/bindings.cpp:654-930).  It
// holds no search logic: every call goes through the C ABI in psb200.h.
// Differences from the reference, all deliberate:
//   * CUDA failures raise RuntimeError (the reference only prints them,
//     fft3.cu:59-91) and there is no CPU fallback;
//   * negative voxel values are rejected with RuntimeError;
//   * the GIL is released while the device works.  The module's two
//     process-wide device contexts (the search context behind the
//     generation cache, and the packing context of pack_native) are each
//     guarded by a mutex instead, so calls from several Python threads are
//     serialised per context as the GIL serialises them in the reference.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <fstream>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/psb200.h"

namespace py = pybind11;

using IntArr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>;

namespace {

constexpr int kINF = 1000000000;  // constants.h:21

struct Grid {
    IntArr arr;
    int n[3];
    const int32_t* ptr() const { return arr.data(); }
};

// numpy_to_flat_grid (bindings.cpp:129-148): forcecast to int32, 3-D only
Grid to_grid(py::handle obj, const char* what = "Input array") {
    IntArr a = IntArr::ensure(obj);
    if (!a) throw std::runtime_error(std::string(what) + " must be convertible to an int32 array");
    if (a.ndim() != 3)
        throw std::runtime_error(std::string(what) + " must be 3-dimensional, got " + std::to_string(a.ndim()) + "D");
    Grid g{a, {(int)a.shape(0), (int)a.shape(1), (int)a.shape(2)}};
    return g;
}

[[noreturn]] void raise_status(int st) {
    char buf[1024];
    psb_last_error(buf, sizeof(buf));
    throw std::runtime_error(std::string(buf[0] ? buf : "psacking_b200 error ") +
                             (buf[0] ? "" : std::to_string(st)));
}

void check(int st) {
    if (st != PSB_OK) raise_status(st);
}

py::array_t<int32_t> new_grid(const int* n) { return py::array_t<int32_t>({n[0], n[1], n[2]}); }

py::tuple result_tuple(const psb_result& r) {
    return py::make_tuple(py::make_tuple(r.x, r.y, r.z), (bool)r.found, r.score);
}

// ---------------------------------------------------------------------------
// the global context + generation cache (fft3.cu:1463, bindings.cpp:209)
// ---------------------------------------------------------------------------
psb_tray* g_ctx = nullptr;
uint64_t g_cached_generation = 0;

// Holds g_ctx_mu for the whole call of a function that reads or changes
// g_ctx, g_ctx_initialized or g_cached_generation, so a tray set up for one
// generation is searched by the same call.  The mutex is only waited for
// with the GIL released (the GIL is taken back once it is held), so a thread
// holding the GIL never waits for it and no two threads can wait on each
// other.  Recursive: the search functions call gpu_tray_is_initialized.
std::recursive_mutex g_ctx_mu;

class CtxLock {
  public:
    CtxLock() : lk_(g_ctx_mu, std::defer_lock) {
        py::gil_scoped_release nogil;
        lk_.lock();
    }

  private:
    std::unique_lock<std::recursive_mutex> lk_;
};

void ctx_init(const Grid& tray, const Grid& phi) {
    if (phi.n[0] != tray.n[0] || phi.n[1] != tray.n[1] || phi.n[2] != tray.n[2])
        throw std::runtime_error("tray_distance must have the tray's shape");
    int dx, dy, dz;
    if (g_ctx) {
        psb_tray_dims(g_ctx, &dx, &dy, &dz);
        if (dx != tray.n[0] || dy != tray.n[1] || dz != tray.n[2]) {
            psb_tray_destroy(g_ctx);
            g_ctx = nullptr;
        }
    }
    int st = PSB_OK;
    {
        py::gil_scoped_release nogil;
        if (!g_ctx) st = psb_tray_create(tray.n[0], tray.n[1], tray.n[2], &g_ctx);
        if (st == PSB_OK) st = psb_tray_set(g_ctx, tray.ptr(), phi.ptr());
    }
    check(st);
}

bool ctx_ready() {
    if (!g_ctx) return false;
    int dx, dy, dz;
    return psb_tray_dims(g_ctx, &dx, &dy, &dz) == PSB_OK;
}

bool g_ctx_initialized = false;

std::vector<Grid> to_grids(py::list orientations) {
    std::vector<Grid> gs;
    gs.reserve(py::len(orientations));
    for (auto o : orientations) gs.push_back(to_grid(o));
    return gs;
}

psb_result search_list(const std::vector<Grid>& gs, int flags) {
    std::vector<const int32_t*> ptrs;
    std::vector<int32_t> dims;
    for (auto& g : gs) {
        ptrs.push_back(g.ptr());
        dims.insert(dims.end(), {g.n[0], g.n[1], g.n[2]});
    }
    psb_result r;
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_tray_search(g_ctx, ptrs.data(), dims.data(), (int)gs.size(), flags, &r, nullptr);
    }
    check(st);
    return r;
}

// ---------------------------------------------------------------------------
// exported functions
// ---------------------------------------------------------------------------
py::tuple py_fft_search_placement(py::handle item, py::handle tray) {
    Grid it = to_grid(item), tr = to_grid(tray);
    psb_result r;
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_fft_search_placement(it.ptr(), it.n[0], it.n[1], it.n[2], tr.ptr(), tr.n[0], tr.n[1], tr.n[2], &r);
    }
    check(st);
    return result_tuple(r);
}

py::tuple py_fft_search_placement_with_cache(py::handle item, py::handle tray, py::handle tray_distance,
                                             uint64_t generation) {
    Grid it = to_grid(item), tr = to_grid(tray), ph = to_grid(tray_distance);
    CtxLock lock;
    if (it.n[0] > tr.n[0] || it.n[1] > tr.n[1] || it.n[2] > tr.n[2])  // bindings.cpp:230-234
        return py::make_tuple(py::make_tuple(-1, -1, -1), false, 0.0);
    if (!g_ctx_initialized || generation != g_cached_generation) {
        ctx_init(tr, ph);
        g_ctx_initialized = true;
        g_cached_generation = generation;
    }
    psb_result r = search_list({it}, PSB_MODE_BLOCK);
    return result_tuple(r);
}

py::tuple py_fft_search_batch(py::list orientations, py::handle tray, py::handle tray_distance, uint64_t generation) {
    Grid tr = to_grid(tray), ph = to_grid(tray_distance);
    CtxLock lock;
    if (!g_ctx_initialized || generation != g_cached_generation) {
        ctx_init(tr, ph);
        g_ctx_initialized = true;
        g_cached_generation = generation;
    }
    auto gs = to_grids(orientations);
    psb_result r = search_list(gs, PSB_MODE_BLOCK);
    // fft3.cu:1558-1560: an unsuccessful batch reports its initial score 1e30
    double score = r.found ? r.score : 1e30;
    return py::make_tuple(py::make_tuple(r.x, r.y, r.z), (bool)r.found, score);
}

py::tuple py_fft_search_batch_interlocking_free(py::list orientations, py::handle tray, py::handle tray_distance,
                                                uint64_t generation) {
    Grid tr = to_grid(tray), ph = to_grid(tray_distance);
    CtxLock lock;
    if (!g_ctx_initialized || generation != g_cached_generation) {
        ctx_init(tr, ph);
        g_ctx_initialized = true;
        g_cached_generation = generation;
    }
    auto gs = to_grids(orientations);
    psb_result r = search_list(gs, PSB_MODE_BLOCK | PSB_FLAG_INTERLOCK);
    double score = r.found ? r.score : 1e30;
    return py::make_tuple(py::make_tuple(r.x, r.y, r.z), (bool)r.found, score, r.found ? r.orientation : -1);
}

py::array_t<int32_t> py_place_in_tray(py::handle item, py::handle tray, py::tuple position, int item_id) {
    Grid it = to_grid(item), tr = to_grid(tray);
    int x = position[0].cast<int>(), y = position[1].cast<int>(), z = position[2].cast<int>();
    auto out = new_grid(tr.n);
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_place_in_tray(it.ptr(), it.n[0], it.n[1], it.n[2], tr.ptr(), tr.n[0], tr.n[1], tr.n[2], x, y, z,
                               item_id, out.mutable_data(), nullptr);
    }
    check(st);
    return out;
}

py::array_t<int32_t> py_dft_conv3(py::handle a, py::handle b) {
    Grid ga = to_grid(a), gb = to_grid(b);
    if (ga.n[0] != gb.n[0] || ga.n[1] != gb.n[1] || ga.n[2] != gb.n[2])
        throw std::runtime_error("Input grids must be of the same size for convolution");
    auto out = new_grid(ga.n);
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_dft_conv3(ga.ptr(), gb.ptr(), ga.n[0], ga.n[1], ga.n[2], out.mutable_data());
    }
    check(st);
    return out;
}

py::array_t<int32_t> py_dft_corr3(py::handle a, py::handle b) {
    Grid ga = to_grid(a), gb = to_grid(b);
    if (ga.n[0] != gb.n[0] || ga.n[1] != gb.n[1] || ga.n[2] != gb.n[2])
        throw std::runtime_error("Input grids must be of the same size for convolution");
    auto out = new_grid(ga.n);
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_dft_corr3(ga.ptr(), gb.ptr(), ga.n[0], ga.n[1], ga.n[2], out.mutable_data());
    }
    check(st);
    return out;
}

py::array_t<int32_t> py_calculate_distance(py::handle grid) {
    Grid g = to_grid(grid);
    auto out = new_grid(g.n);
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_calculate_distance(g.ptr(), g.n[0], g.n[1], g.n[2], out.mutable_data());
    }
    check(st);
    return out;
}

py::array_t<int32_t> py_collision_grid(py::handle tray, py::handle item) {
    Grid tr = to_grid(tray), it = to_grid(item);
    auto out = new_grid(tr.n);
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_collision_grid(tr.ptr(), tr.n[0], tr.n[1], tr.n[2], it.ptr(), it.n[0], it.n[1], it.n[2],
                                out.mutable_data());
    }
    check(st);
    return out;
}

py::array_t<int32_t> py_interlocking_free_positions(py::handle tray, py::handle obj) {
    Grid tr = to_grid(tray, "Tray array"), ob = to_grid(obj, "Object array");
    auto out = new_grid(tr.n);
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_interlocking_free_positions(tr.ptr(), tr.n[0], tr.n[1], tr.n[2], ob.ptr(), ob.n[0], ob.n[1], ob.n[2],
                                             out.mutable_data());
    }
    check(st);
    return out;
}

// get_voxel_grid_bounds (voxelGrid.cpp:279-299): host scan, (INF..)/(-INF..) when empty
std::pair<std::tuple<int, int, int>, std::tuple<int, int, int>> bounds_of(const Grid& g) {
    int lo[3] = {kINF, kINF, kINF}, hi[3] = {-kINF, -kINF, -kINF};
    const int32_t* p = g.ptr();
    for (int i = 0; i < g.n[0]; ++i)
        for (int j = 0; j < g.n[1]; ++j)
            for (int k = 0; k < g.n[2]; ++k)
                if (p[((size_t)i * g.n[1] + j) * g.n[2] + k] > 0) {
                    int c[3] = {i, j, k};
                    for (int a = 0; a < 3; ++a) {
                        lo[a] = std::min(lo[a], c[a]);
                        hi[a] = std::max(hi[a], c[a]);
                    }
                }
    return {{lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}};
}

py::tuple py_get_bounds(py::handle grid) {
    Grid g = to_grid(grid);
    auto b = bounds_of(g);
    auto [lx, ly, lz] = b.first;
    auto [hx, hy, hz] = b.second;
    return py::make_tuple(py::make_tuple(lx, ly, lz), py::make_tuple(hx, hy, hz));
}

py::array_t<int32_t> py_make_tight(py::handle grid) {
    Grid g = to_grid(grid);
    auto b = bounds_of(g);
    auto [lx, ly, lz] = b.first;
    auto [hx, hy, hz] = b.second;
    if (hx == -kINF)  // voxelGrid.cpp:228-229 raise() -> invalid_argument -> ValueError
        throw py::value_error("(make_voxel_grid_tight) Voxel grid doesn't have any occupied cells");
    int n[3] = {hx - lx + 1, hy - ly + 1, hz - lz + 1};
    auto out = new_grid(n);
    int32_t* o = out.mutable_data();
    const int32_t* p = g.ptr();
    for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
            std::memcpy(&o[((size_t)i * n[1] + j) * n[2]], &p[((size_t)(i + lx) * g.n[1] + (j + ly)) * g.n[2] + lz],
                        sizeof(int32_t) * n[2]);
    return out;
}

void py_gpu_tray_init(py::handle tray, py::handle tray_distance) {
    Grid tr = to_grid(tray), ph = to_grid(tray_distance);
    CtxLock lock;
    ctx_init(tr, ph);
    g_ctx_initialized = true;
}

void py_gpu_tray_cleanup() {
    CtxLock lock;
    if (g_ctx) psb_tray_destroy(g_ctx);
    g_ctx = nullptr;
    g_ctx_initialized = false;
}

bool py_gpu_tray_is_initialized() {
    CtxLock lock;
    return g_ctx_initialized && ctx_ready();
}

py::tuple py_gpu_tray_search(py::handle item) {
    CtxLock lock;
    if (!py_gpu_tray_is_initialized())
        throw std::runtime_error("GPU tray context not initialized. Call gpu_tray_init() first.");
    Grid it = to_grid(item);
    psb_result r = search_list({it}, PSB_MODE_BLOCK);
    return result_tuple(r);
}

// Device-resident greedy loop used by psacking_b200.BinPacker (see psb_pack).
// cells > 0 of every item (BinPacker's volumes, packer.py: np.sum(item > 0)),
// items spread over the host cores
py::list py_positive_counts(py::list items) {
    auto gs = to_grids(items);
    std::vector<const int32_t*> ptrs;
    std::vector<size_t> sizes;
    for (auto& g : gs) {
        ptrs.push_back(g.ptr());
        sizes.push_back((size_t)g.n[0] * g.n[1] * g.n[2]);
    }
    std::vector<long long> out(gs.size(), 0);
    {
        py::gil_scoped_release nogil;
        std::atomic<size_t> next(0);
        auto work = [&]() {
            for (size_t i = next.fetch_add(1); i < ptrs.size(); i = next.fetch_add(1)) {
                const int32_t* a = ptrs[i];
                const size_t m = sizes[i];
                long long c = 0;
                for (size_t k = 0; k < m; ++k) c += a[k] > 0;
                out[i] = c;
            }
        };
        const int nthr = (int)std::min<size_t>(gs.size() / 16 + 1, std::max(1u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        for (int w = 1; w < nthr; ++w) pool.emplace_back(work);
        work();
        for (auto& th : pool) th.join();
    }
    py::list r;
    for (long long c : out) r.append(c);
    return r;
}

py::tuple py_pack_native(py::list items, py::handle initial_tray, py::array_t<int32_t> orient_maps, bool interlock,
                         int id_offset) {
    Grid tr = to_grid(initial_tray);
    auto gs = to_grids(items);
    std::vector<const int32_t*> ptrs;
    std::vector<int32_t> dims;
    for (auto& g : gs) {
        ptrs.push_back(g.ptr());
        dims.insert(dims.end(), {g.n[0], g.n[1], g.n[2]});
    }
    auto maps = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(orient_maps);
    if (maps.ndim() != 2 || maps.shape(1) != 6) throw std::runtime_error("orient_maps must be (n, 6) int32");
    int n_orient = (int)maps.shape(0);
    std::vector<psb_result> res(gs.size());
    auto out = new_grid(tr.n);
    int st;
    long long occupied = 0;
    int32_t lo[3] = {-1, -1, -1}, hi[3] = {-1, -1, -1};
    {
        // the packing context (about 90 MB per orientation slot) is kept for
        // the next run with the same tray shape instead of being rebuilt
        py::gil_scoped_release nogil;
        static psb_tray* pack_ctx = nullptr;
        static std::mutex pack_mu;  // one run at a time on the shared context (GIL released here)
        std::lock_guard<std::mutex> lk(pack_mu);
        if (pack_ctx) {
            int dx, dy, dz;
            psb_tray_dims(pack_ctx, &dx, &dy, &dz);
            if (dx != tr.n[0] || dy != tr.n[1] || dz != tr.n[2]) {
                psb_tray_destroy(pack_ctx);
                pack_ctx = nullptr;
            }
        }
        st = pack_ctx ? PSB_OK : psb_tray_create(tr.n[0], tr.n[1], tr.n[2], &pack_ctx);
        if (st == PSB_OK) st = psb_tray_set(pack_ctx, tr.ptr(), nullptr);
        if (st == PSB_OK)
            st = psb_pack(pack_ctx, ptrs.data(), dims.data(), (int)gs.size(), maps.data(), n_orient,
                          interlock ? 1 : 0, id_offset, res.data(), out.mutable_data());
        if (st == PSB_OK) st = psb_tray_stats(pack_ctx, &occupied, lo, hi);
    }
    check(st);
    py::list pl;
    for (auto& r : res)
        pl.append(py::make_tuple(py::make_tuple(r.x, r.y, r.z), (bool)r.found, r.score, r.orientation, r.diag,
                                 r.n_candidates, r.err_ratio));
    // the final tray's occupied cells and bounding box, counted on the device
    py::tuple stats = py::make_tuple(occupied, py::make_tuple(lo[0], lo[1], lo[2]), py::make_tuple(hi[0], hi[1], hi[2]));
    return py::make_tuple(out, pl, stats);
}

// trays: list of (dims, [items in packing order]) -> list of (final tray, placements)
py::list py_pack_many(py::list trays, py::array_t<int32_t> orient_maps, bool interlock, int concurrency) {
    auto maps = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(orient_maps);
    if (maps.ndim() != 2 || maps.shape(1) != 6) throw std::runtime_error("orient_maps must be (n, 6) int32");
    const int n_orient = (int)maps.shape(0);
    std::vector<Grid> grids;
    std::vector<const int32_t*> ptrs;
    std::vector<int32_t> idims, tdims, counts;
    for (auto tr : trays) {
        py::tuple tt = tr.cast<py::tuple>();
        py::tuple d = tt[0].cast<py::tuple>();
        for (int a = 0; a < 3; ++a) tdims.push_back(d[a].cast<int>());
        py::list its = tt[1].cast<py::list>();
        counts.push_back((int)py::len(its));
        for (auto it : its) grids.push_back(to_grid(it));
    }
    for (auto& g : grids) {
        ptrs.push_back(g.ptr());
        idims.insert(idims.end(), {g.n[0], g.n[1], g.n[2]});
    }
    const int n_trays = (int)counts.size();
    std::vector<psb_result> res(grids.size());
    std::vector<py::array_t<int32_t>> outs;
    std::vector<int32_t*> outp;
    for (int i = 0; i < n_trays; ++i) {
        outs.push_back(new_grid(&tdims[3 * i]));
        outp.push_back(outs.back().mutable_data());
    }
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_pack_many(n_trays, tdims.data(), ptrs.data(), idims.data(), counts.data(), maps.data(), n_orient,
                           interlock ? 1 : 0, concurrency, res.data(), outp.data());
    }
    check(st);
    py::list out;
    size_t k = 0;
    for (int i = 0; i < n_trays; ++i) {
        py::list pl;
        for (int j = 0; j < counts[i]; ++j, ++k) {
            const psb_result& r = res[k];
            pl.append(py::make_tuple(py::make_tuple(r.x, r.y, r.z), (bool)r.found, r.score, r.orientation, r.diag,
                                     r.n_candidates, r.err_ratio));
        }
        out.append(py::make_tuple(outs[i], pl));
    }
    return out;
}

py::dict py_search_detail(py::list orientations, int flags, bool per_orientation) {
    CtxLock lock;
    if (!py_gpu_tray_is_initialized()) throw std::runtime_error("GPU tray context not initialized");
    auto gs = to_grids(orientations);
    std::vector<const int32_t*> ptrs;
    std::vector<int32_t> dims;
    for (auto& g : gs) {
        ptrs.push_back(g.ptr());
        dims.insert(dims.end(), {g.n[0], g.n[1], g.n[2]});
    }
    psb_result best;
    std::vector<psb_result> per(gs.size());
    int st;
    {
        py::gil_scoped_release nogil;
        st = psb_tray_search(g_ctx, ptrs.data(), dims.data(), (int)gs.size(), flags, &best,
                             per_orientation ? per.data() : nullptr);
    }
    check(st);
    py::list pl;
    if (per_orientation)
        for (auto& r : per)
        pl.append(py::make_tuple(py::make_tuple(r.x, r.y, r.z), (bool)r.found, r.score, r.diag, r.n_candidates,
                                 r.err_ratio));
    py::dict d;
    d["best"] = py::make_tuple(py::make_tuple(best.x, best.y, best.z), (bool)best.found, best.score, best.orientation);
    d["best_diag"] = best.diag;
    d["per_orientation"] = pl;
    return d;
}

int py_device_count() {
    int n = 0;
    psb_device_count(&n);
    return n;
}

// bindings.cpp:285-302 and 304-313: the STL reader and the .vox encoder live
// in the package's Python modules (psacking_b200.voxelize, psacking_b200.vox);
// the rasterization itself is psb_voxelize_mesh.  These keep the module's
// export list equal to the reference's.
py::object py_voxelize_stl(py::object path, int resolution) {
    return py::module_::import("psacking_b200.voxelize").attr("voxelize_stl")(path, resolution);
}

void py_save_vox(py::object grid, py::object path) {
    py::module_::import("psacking_b200.vox").attr("save_vox")(grid, path);
}

}  // namespace

PYBIND11_MODULE(_core, m) {
    m.doc() = "B200 placement-search engine; drop-in for spectral_packer._core (spectral_packing/bindings.cpp).";
    m.def("fft_search_placement", &py_fft_search_placement, py::arg("item"), py::arg("tray"));
    m.def("fft_search_placement_with_cache", &py_fft_search_placement_with_cache, py::arg("item"), py::arg("tray"),
          py::arg("tray_distance"), py::arg("generation"));
    m.def("place_in_tray", &py_place_in_tray, py::arg("item"), py::arg("tray"), py::arg("position"),
          py::arg("item_id") = 1);
    m.def("dft_conv3", &py_dft_conv3, py::arg("a"), py::arg("b"));
    m.def("dft_corr3", &py_dft_corr3, py::arg("a"), py::arg("b"));
    m.def("calculate_distance", &py_calculate_distance, py::arg("grid"),
          "L1 distance field to voxels equal to 1 (the reference's tests pin L1).");
    m.def("collision_grid", &py_collision_grid, py::arg("tray"), py::arg("item"));
    m.def("make_tight", &py_make_tight, py::arg("grid"));
    m.def("get_bounds", &py_get_bounds, py::arg("grid"));
    m.def("gpu_tray_init", &py_gpu_tray_init, py::arg("tray"), py::arg("tray_distance"));
    m.def("gpu_tray_cleanup", &py_gpu_tray_cleanup);
    m.def("gpu_tray_is_initialized", &py_gpu_tray_is_initialized);
    m.def("gpu_tray_search", &py_gpu_tray_search, py::arg("item"));
    m.def("fft_search_batch", &py_fft_search_batch, py::arg("orientations"), py::arg("tray"),
          py::arg("tray_distance"), py::arg("generation"));
    m.def("fft_search_batch_interlocking_free", &py_fft_search_batch_interlocking_free, py::arg("orientations"),
          py::arg("tray"), py::arg("tray_distance"), py::arg("generation"));
    m.def("interlocking_free_positions", &py_interlocking_free_positions, py::arg("tray"), py::arg("obj"));
    // engine extensions (not in the reference module)
    m.def("positive_counts", &py_positive_counts, py::arg("items"),
          "Number of cells > 0 of each int32 grid (on all host cores).");
    m.def("pack_native", &py_pack_native, py::arg("items"), py::arg("initial_tray"), py::arg("orient_maps"),
          py::arg("interlock"), py::arg("id_offset"));
    m.def("search_detail", &py_search_detail, py::arg("orientations"), py::arg("flags"),
          py::arg("per_orientation") = true,
          "Search the initialised tray.  per_orientation=True: every orientation's own result (interlocking "
          "searches run the flood fill for all of them); False: only the best (lazy flood fill).");
    m.def("pack_many", &py_pack_many, py::arg("trays"), py::arg("orient_maps"), py::arg("interlock"),
          py::arg("concurrency") = 8);
    m.def("voxelize_stl", &py_voxelize_stl, py::arg("path"), py::arg("resolution") = 128,
          "Surface voxels of an STL mesh, tight int32 grid (GPU rasterizer).");
    m.def("save_vox", &py_save_vox, py::arg("grid"), py::arg("path"),
          "Save a voxel grid in the reference's .vox layout.");
    m.def("device_count", &py_device_count);
    m.def("set_fast_fft", [](bool on) { psb_set_fast_fft(on ? 1 : 0); }, py::arg("on"),
          "Use the specialised two-pass FFT kernels where a plan exists (default) or force the generic path.");
    m.def("set_cand_filter", [](bool on) { check(psb_set_cand_filter(on ? 1 : 0)); }, py::arg("on"),
          "Candidate pre-filter of the packing loop (default on; same placements either way).");
    m.def("set_direct_max", [](int n) { check(psb_set_direct_max(n)); }, py::arg("n"),
          "Candidate limit below which the packing loop decides an orientation without transforms.");
    m.def("set_filter_cut", [](int pct) { check(psb_set_filter_cut(pct)); }, py::arg("pct"),
          "Pre-filter cut-off percentage (default 50, 0 off; same placements either way).");
    m.def("set_share_flips", [](bool on) { check(psb_set_share_flips(on ? 1 : 0)); }, py::arg("on"),
          "Share the z,y transforms among the flips of each axis permutation, or transform each orientation on "
          "its own (the default).");
    m.def("set_plane_variant", [](int v) { check(psb_set_plane_variant(v)); }, py::arg("variant"),
          "Plane-pass kernel for the specialised lengths: 3 (warp-owned lines, default) or 2.");
    m.def("set_late_direct_max", [](int n) { check(psb_set_late_direct_max(n)); }, py::arg("n"),
          "Ok-cell limit below which an orientation skips the proximity transforms (0 off; same placements).");
    m.def("set_uf_limit", [](int n) { check(psb_set_uf_limit(n)); }, py::arg("n"),
          "Union-find step bound of the flood fill (n <= 0: the default); past it searches raise.");
    m.def("debug_fail_alloc", [](int n) { check(psb_debug_fail_alloc(n)); }, py::arg("n"),
          "Test hook: the n-th device allocation from now fails (0 disarms).");
    m.def("debug_live_allocs", []() {
        long long n = 0;
        check(psb_debug_live_allocs(&n));
        return n;
    }, "Test hook: the engine's device allocations not yet freed.");
    m.attr("VOXEL_RESOLUTION") = 128;
    m.attr("HEIGHT_PENALTY") = 100000000.0;
    m.attr("__version__") = "0.1.0";
    m.attr("MODE_SCAN") = PSB_MODE_SCAN;
    m.attr("MODE_BLOCK") = PSB_MODE_BLOCK;
    m.attr("FLAG_INTERLOCK") = PSB_FLAG_INTERLOCK;
}
