// Batch planner: validates pairs, lays out the workspace, builds the work
// queue of (pair, path, scanline-group) units and issues the launches.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>

#include "vx_internal.hpp"

namespace vxsgm {

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v, size_t a = kAlign) { return (v + a - 1) / a * a; }

// Path directions in slab order; the first two are the reference's
// (vx-vision/src/kernels/sgm.rs:197-200), the rest are the 4/8-path extension.
const int kDirs[8][2] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}, {1, 1}, {-1, 1}, {1, -1}, {-1, -1}};

}  // namespace

int census_bits(const vx_sgm_config& cfg) {
    return (int)((2 * cfg.census_radius_x + 1) * (2 * cfg.census_radius_y + 1)) - 1;
}

// Slab format of a configuration. A path cost is at most the matching cost
// (<= 64: census bits or the border cost) plus P2 unless it wraps below zero,
// so byte vectors hold nearly every vector when 64 + P2 <= 254; otherwise most
// vectors would escape and u16 slabs alone are smaller and read faster.
// VX_SGM_SLAB_FORMAT=bytes|wide forces one format (both are exact for every
// configuration; the tests run each on the other's configurations).
bool wide_slabs(const vx_sgm_config& c) {
    if (const char* f = std::getenv("VX_SGM_SLAB_FORMAT")) {
        if (std::strcmp(f, "bytes") == 0) return false;
        if (std::strcmp(f, "wide") == 0) return true;
    }
    return 64 + (int)(uint16_t)c.p2 > 254;
}

uint32_t shadow_pool_vectors(uint32_t width, uint32_t height, const vx_sgm_config& cfg) {
    if (const char* f = std::getenv("VX_SGM_SHADOW_POOL")) {
        const long v = std::strtol(f, nullptr, 10);
        if (v > 0) return (uint32_t)v;
    }
    const size_t vectors = (size_t)width * height * cfg.num_paths;
    return (uint32_t)std::max<size_t>(1024, (vectors + 15) / 16);
}

size_t pair_workspace_bytes(uint32_t width, uint32_t height, const vx_sgm_config& cfg,
                            size_t census_word_bytes, bool compact_shadow) {
    const size_t npx = (size_t)width * height, ct = census_word_bytes, P = cfg.num_paths;
    const size_t dp = (cfg.num_disparities + 7) / 8 * 8;
    const size_t dv = (cfg.num_disparities + 15) / 16 * 16;
    const size_t banded = (size_t)((height + 31) / 32) * 32 * width * ct;
    const size_t guard = kCensusGuardWords * ct;
    const bool wide = wide_slabs(cfg);
    const size_t bytes = wide ? 0 : align_up(npx * dv * P);
    const size_t shadow_vectors = (compact_shadow && !wide) ? shadow_pool_vectors(width, height, cfg) : npx * P;
    return 2 * align_up(npx * ct + 2 * guard) + 2 * align_up(banded) + bytes +
           align_up(shadow_vectors * dp * sizeof(uint16_t));
}

size_t pair_cost_bytes(uint32_t width, uint32_t height, const vx_sgm_config& cfg) {
    return align_up((size_t)width * height * ((cfg.num_disparities + 15) / 16 * 16));
}

size_t pair_table_bytes_bound(uint32_t width, uint32_t height, const vx_sgm_config& cfg) {
    const size_t P = cfg.num_paths;
    // Units of the scan form hold the fewest scanlines (ScanGeometry::scanlines, 1..16).
    const size_t per_unit = (size_t)scan_geometry((cfg.num_disparities + 15) / 16 * 16).scanlines;
    const size_t units = P * (((size_t)width + height - 1 + per_unit - 1) / per_unit);
    return sizeof(PairDev) + P * sizeof(JobDev) + units * sizeof(UnitDev) + sizeof(unsigned) +
           4 * kAlign;
}

void rebind_pointers(Plan& plan, const std::vector<PairSpec>& specs) {
    for (size_t i = 0; i < specs.size(); ++i) {
        PairDev& pd = plan.pairs[i];
        const PairSpec& s = specs[i];
        pd.left = static_cast<const uint8_t*>(s.left->ptr);
        pd.right = static_cast<const uint8_t*>(s.right->ptr);
        pd.left_pitch = s.left->pitch;
        pd.right_pitch = s.right->pitch;
        pd.out_f32 = static_cast<float*>(s.out_f32->ptr);
        pd.out_f32_pitch = s.out_f32->pitch;
        pd.out_i16 = s.out_i16 ? static_cast<int16_t*>(s.out_i16->ptr) : nullptr;
        pd.out_i16_pitch = s.out_i16 ? s.out_i16->pitch : 0;
        pd.out_depth = s.out_depth ? static_cast<float*>(s.out_depth->ptr) : nullptr;
        pd.out_depth_pitch = s.out_depth ? s.out_depth->pitch : 0;
        pd.depth_scale = s.depth_scale;
        pd.depth_invalid = s.depth_invalid;
    }
}

vx_status validate_pair(const PairSpec& p) {
    if (!p.left || !p.right || !p.out_f32)
        return fail(VX_ERR_INVALID_ARGUMENT, "left, right and output images are required");
    if (p.left->format != VX_FORMAT_U8 || p.right->format != VX_FORMAT_U8)
        return fail(VX_ERR_INVALID_ARGUMENT, "input images must be U8");
    if (p.out_f32->format != VX_FORMAT_F32)
        return fail(VX_ERR_INVALID_ARGUMENT, "output image must be F32");
    if (p.out_i16 && p.out_i16->format != VX_FORMAT_I16)
        return fail(VX_ERR_INVALID_ARGUMENT, "integer output image must be I16");
    if (p.out_depth && p.out_depth->format != VX_FORMAT_F32)
        return fail(VX_ERR_INVALID_ARGUMENT, "depth output image must be F32");
    const uint32_t w = p.left->width, h = p.left->height;
    if (p.right->width != w || p.right->height != h || p.out_f32->width != w ||
        p.out_f32->height != h || (p.out_i16 && (p.out_i16->width != w || p.out_i16->height != h)) ||
        (p.out_depth && (p.out_depth->width != w || p.out_depth->height != h)))
        return fail(VX_ERR_SIZE_MISMATCH, "texture size mismatch");
    if (w > (uint32_t)kMaxWidth)
        return fail(VX_ERR_INVALID_CONFIG, "image width %u exceeds %d", w, kMaxWidth);
    const vx_sgm_config& c = p.cfg;
    if (c.num_disparities < 1 || c.num_disparities > 256)
        return fail(VX_ERR_INVALID_CONFIG, "num_disparities %u not in 1..256", c.num_disparities);
    if (!(c.p1 >= 0.0f && c.p1 < 65536.0f) || !(c.p2 >= 0.0f && c.p2 < 65536.0f))
        return fail(VX_ERR_INVALID_CONFIG, "p1/p2 must be in [0, 65536)");
    if (c.census_radius_x > 31 || c.census_radius_y > 31 || census_bits(c) > 64)
        return fail(VX_ERR_INVALID_CONFIG, "census window %ux%u exceeds 64 bits",
                    2 * c.census_radius_x + 1, 2 * c.census_radius_y + 1);
    if (c.num_paths != 2 && c.num_paths != 4 && c.num_paths != 8)
        return fail(VX_ERR_INVALID_CONFIG, "num_paths must be 2, 4 or 8");
    return VX_OK;
}

// The aggregation launch shape of a plan whose units are in longest-first
// order, and the queue classes that go with it (units reordered class by
// class, longest-first inside each class).
//  * Single-scanline form: one queue; `warpgroups` or the default count.
//  * Scanline-pair form: warpgroups with per-class TMEM column budgets
//    (pairs::budgets_for); class c holds the units whose padded D is at most
//    the c-th largest budget and above the next one. With one budget value
//    there is one class and the order stays plainly longest-first.
template <typename CostFn>
vx_status plan_queues(Plan& pl, int warpgroups, CostFn unit_cost) {
    AggLaunch& L = pl.agg;
    L = AggLaunch{};
    AggQueues& q = L.queues;
    const int nu = (int)pl.units.size();
    auto unit_dp = [&](const UnitDev& u) { return pl.pairs[pl.jobs[u.job].pair].nd_pad; };
    if (pl.unit_scanlines == kScanForm) {      // one queue, warps per SM by occupancy
        L.warpgroups = 1;
        q.n_classes = 1;
        q.begin[1] = nu;
        for (int c = 2; c <= kMaxQueueClasses; ++c) q.begin[c] = nu;
        return VX_OK;
    }
    if (pl.unit_scanlines != kUnitScanlines) {
        const int wmax = single::max_warpgroups(pl.dp_max, pl.census64);
        L.warpgroups = warpgroups > 0 ? std::min(warpgroups, wmax)
                                      : single::default_warpgroups(pl.dp_max, pl.census64, nu);
        q.n_classes = 1;
        q.begin[1] = nu;
        for (int w = 0; w < L.warpgroups; ++w) q.col0[w] = w * (pl.dp_max / 2);
        return VX_OK;
    }
    // Distinct padded D of the units (descending) and their shares of the work.
    std::vector<int> dps;
    std::vector<double> work;
    {
        std::map<int, double, std::greater<int>> w;
        for (const UnitDev& u : pl.units) w[unit_dp(u)] += (double)unit_cost(u);
        for (const auto& kv : w) {
            dps.push_back(kv.first);
            work.push_back(kv.second);
        }
    }
    if (dps.empty()) {
        dps.push_back(pl.dp_max);
        work.push_back(1.0);
    }
    const int nd = (int)dps.size();
    const int wmax = pairs::max_warpgroups(dps[0], dps[nd - 1], pl.wide_tiles);
    double path_pd = 0.0;
    for (const PairDev& p : pl.pairs) path_pd += (double)p.width * p.height * p.nd * p.num_paths;
    const double chain = nu > 0 ? (double)unit_cost(pl.units[0]) : 0.0;   // units are longest-first
    int wg = warpgroups > 0 ? std::min(warpgroups, wmax)
                            : pairs::default_warpgroups(dps.data(), work.data(), nd, pl.wide_tiles, path_pd, chain);
    int cols[kAggMaxWarpgroups] = {};
    while (wg > 1 && pairs::budgets_for(dps.data(), work.data(), nd, wg, cols) <= 0.0) --wg;
    if (wg == 1) cols[0] = dps[0];
    L.warpgroups = wg;
    // Classes: the distinct budgets, largest first (at most kAggMaxWarpgroups <= kMaxQueueClasses).
    std::vector<int> cls;
    for (int w = 0; w < wg; ++w)
        if (cls.empty() || cls.back() != cols[w]) cls.push_back(cols[w]);
    q.n_classes = (int)cls.size();
    int sum = 0;
    for (int w = 0; w < wg; ++w) {
        q.col0[w] = sum;
        sum += cols[w];
        q.first_class[w] = (int)(std::find(cls.begin(), cls.end(), cols[w]) - cls.begin());
    }
    L.tmem_cols = 32;
    while (L.tmem_cols < sum) L.tmem_cols <<= 1;
    if (L.tmem_cols > 512) return fail(VX_ERR_GPU, "planner: TMEM budgets of %d columns exceed 512", sum);
    // Class of a unit: the last class whose budget still holds its padded D.
    auto class_of = [&](const UnitDev& u) {
        const int dp = unit_dp(u);
        int c = 0;
        while (c + 1 < (int)cls.size() && cls[c + 1] >= dp) ++c;
        return c;
    };
    std::stable_sort(pl.units.begin(), pl.units.end(),
                     [&](const UnitDev& a, const UnitDev& b) { return class_of(a) < class_of(b); });
    for (int c = 0, i = 0; c < q.n_classes; ++c) {
        q.begin[c] = i;
        while (i < nu && class_of(pl.units[i]) == c) ++i;
        q.begin[c + 1] = i;
    }
    for (int c = q.n_classes + 1; c <= kMaxQueueClasses; ++c) q.begin[c] = nu;
    return VX_OK;
}

vx_status build_plan(const std::vector<PairSpec>& specs, Plan* plan, int unit_scanlines, int warpgroups) {
    Plan& pl = *plan;
    pl = Plan{};
    const int n = (int)specs.size();
    for (const auto& s : specs) {
        vx_status st = validate_pair(s);
        if (st != VX_OK) return st;
        if (census_bits(s.cfg) > 32) pl.census64 = true;
    }
    const size_t ct = pl.census64 ? 8 : 4;

    pl.pairs.resize(n);
    pl.pair_data_off.resize(n);
    size_t data = 0;
    int tiles = 0, rows = 0;
    std::vector<UnitDev> units;
    for (int i = 0; i < n; ++i) {
        const PairSpec& s = specs[i];
        const vx_sgm_config& c = s.cfg;
        const int W = (int)s.left->width, H = (int)s.left->height;
        const int D = (int)c.num_disparities, Dp = (D + 7) / 8 * 8, Dv = (D + 15) / 16 * 16;
        const int P = (int)c.num_paths;
        PairDev& pd = pl.pairs[i];
        std::memset(&pd, 0, sizeof pd);
        pd.left = static_cast<const uint8_t*>(s.left->ptr);
        pd.right = static_cast<const uint8_t*>(s.right->ptr);
        pd.left_pitch = s.left->pitch;
        pd.right_pitch = s.right->pitch;
        pd.out_f32 = static_cast<float*>(s.out_f32->ptr);
        pd.out_f32_pitch = s.out_f32->pitch;
        pd.out_i16 = s.out_i16 ? static_cast<int16_t*>(s.out_i16->ptr) : nullptr;
        pd.out_i16_pitch = s.out_i16 ? s.out_i16->pitch : 0;
        pd.out_depth = s.out_depth ? static_cast<float*>(s.out_depth->ptr) : nullptr;
        pd.out_depth_pitch = s.out_depth ? s.out_depth->pitch : 0;
        pd.depth_scale = s.depth_scale;
        pd.depth_invalid = s.depth_invalid;
        pd.width = W;
        pd.height = H;
        pd.nd = D;
        pd.nd_pad = Dp;
        pd.nd_vec = Dv;
        pd.num_paths = P;
        pd.p1 = (int)(uint16_t)c.p1;  // ushort(params.p1), SGMStereo.metal:155
        pd.p2 = (int)(uint16_t)c.p2;
        pd.rx = (int)c.census_radius_x;
        pd.ry = (int)c.census_radius_y;
        pd.subpixel = c.subpixel ? 1 : 0;
        pd.lr_check = c.lr_check ? 1 : 0;
        pd.lr_tolerance = (int)c.lr_tolerance;
        pd.invalid_value = c.invalid_value;
        pd.census_tile_begin = tiles;
        pd.row_begin = rows;
        tiles += 2 * ((W + kCensusTileW - 1) / kCensusTileW) * ((H + kCensusTileH - 1) / kCensusTileH);
        rows += H;
        pl.max_width = std::max(pl.max_width, W);
        pl.max_rx = std::max(pl.max_rx, pd.rx);
        pl.max_ry = std::max(pl.max_ry, pd.ry);

        // Workspace-relative data: 4 census planes, P byte slabs, P shadow slabs
        // (the layout pair_workspace_bytes sizes).
        const size_t npx = (size_t)W * H;
        pl.pair_data_off[i] = data;
        const size_t data0 = data;
        const size_t guard = kCensusGuardWords * ct;
        const size_t cplane = align_up(npx * ct + 2 * guard);                  // guarded row-major
        const size_t bplane = align_up((size_t)((H + 31) / 32) * 32 * W * ct);  // banded copy
        pd.census_l = reinterpret_cast<void*>(data + guard);
        pd.census_r = reinterpret_cast<void*>(data + cplane + guard);
        pd.census_lt = reinterpret_cast<void*>(data + 2 * cplane);
        pd.census_rt = reinterpret_cast<void*>(data + 2 * cplane + bplane);
        data += 2 * cplane + 2 * bplane;
        pd.wide_slabs = wide_slabs(c) ? 1 : 0;
        if (pd.wide_slabs) pl.wide_tiles = true;
        pd.slab_stride = pd.wide_slabs ? 0 : npx * (size_t)Dv;
        pd.slabs = reinterpret_cast<uint8_t*>(data);
        data += align_up(pd.slab_stride * P);
        pd.shadow_stride = npx * (size_t)Dp;
        pd.shadow = reinterpret_cast<uint16_t*>(data);
        if ((size_t)P * npx >= kNoSlot)
            return fail(VX_ERR_INVALID_ARGUMENT, "pair %d: %zu path vectors exceed the 32-bit shadow slots", i,
                        (size_t)P * npx);
        const bool compact = s.compact_shadow && !pd.wide_slabs;
        pd.shadow_cap = compact ? shadow_pool_vectors((uint32_t)W, (uint32_t)H, c) : 0u;
        if (compact) pl.compact = true;
        data += align_up((compact ? (size_t)pd.shadow_cap : npx * P) * Dp * sizeof(uint16_t));
        if (data - data0 != pair_workspace_bytes((uint32_t)W, (uint32_t)H, c, ct, compact))
            return fail(VX_ERR_GPU, "planner: pair layout and its size formula disagree");

        pl.dp_max = std::max(pl.dp_max, Dp);
        pl.dp_min = i == 0 ? Dp : std::min(pl.dp_min, Dp);
        for (int p = 0; p < P; ++p) {
            JobDev j{};
            j.pair = i;
            j.path = p;
            j.dx = kDirs[p][0];
            j.dy = kDirs[p][1];
            j.num_scanlines = j.dy == 0 ? H : (j.dx == 0 ? W : W + H - 1);
            j.k_min = (j.dx > 0 && j.dy != 0) ? -(H - 1) : 0;
            pl.jobs.push_back(j);
        }
    }
    pl.total_tiles = tiles;
    pl.total_rows = rows;
    // The WTA launch's order: the pairs grouped by the WTA row-loop variant
    // (path count, lane form), batch order inside a group, so that the CTAs
    // resident at once mostly run one variant's code.
    {
        std::vector<int> ord(n);
        for (int i = 0; i < n; ++i) ord[i] = i;
        auto variant = [&](int i) {
            const PairDev& q = pl.pairs[i];
            return wta_variant(q.num_paths, q.nd_vec, q.wide_slabs != 0);
        };
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return variant(a) < variant(b); });
        int r = 0;
        for (int k = 0; k < n; ++k) {
            pl.pairs[k].wta_pair = ord[k];
            pl.pairs[k].wta_row_begin = r;
            r += pl.pairs[ord[k]].height;
        }
    }

    // Unit size, i.e. aggregation form: few units (a single pair, small batches)
    // run the across-lanes scan kernel, a segment of lanes per scanline; larger
    // batches the scanline-pair kernel (fewest instructions per path-pd). The
    // single-scanline kernel runs when the autotuner picked it for the batch's
    // key or VX_SGM_AGG_FORM asks for it.
    long long units64 = 0;
    pl.units32 = 0;
    for (const JobDev& j : pl.jobs) {
        units64 += (j.num_scanlines + kUnitScanlines - 1) / kUnitScanlines;
        pl.units32 += (j.num_scanlines + 31) / 32;
    }
    if (unit_scanlines == kUnitScanlines || unit_scanlines == 32 || unit_scanlines == kScanForm)
        pl.unit_scanlines = unit_scanlines;        // the autotuned form
    else
        pl.unit_scanlines = units64 >= kPairKernelMinUnits ? kUnitScanlines
                            : units64 < kScanFormMaxUnits  ? kScanForm
                                                           : 32;
    // VX_SGM_AGG_FORM=pairs|single|scan forces one form (all are exact; the tests
    // run every case through each).
    if (const char* f = std::getenv("VX_SGM_AGG_FORM")) {
        if (std::strcmp(f, "pairs") == 0) pl.unit_scanlines = kUnitScanlines;
        if (std::strcmp(f, "single") == 0) pl.unit_scanlines = 32;
        if (std::strcmp(f, "scan") == 0) pl.unit_scanlines = kScanForm;
    }
    for (int job = 0; job < (int)pl.jobs.size(); ++job) {
        const int per_unit = pl.unit_scanlines == kScanForm
                                 ? scan_geometry(pl.pairs[pl.jobs[job].pair].nd_vec).scanlines
                                 : pl.unit_scanlines;
        for (int k = 0; k < pl.jobs[job].num_scanlines; k += per_unit) units.push_back({job, k});
    }
    // The scanline-pair and scan kernels read the matching costs from a per-pair
    // byte volume (cost.cu), laid out after every pair's census, slab and shadow
    // region; the single-scanline kernel forms them from the census words.
    if (pl.unit_scanlines != 32)
        for (int i = 0; i < n; ++i) {
            PairDev& pd = pl.pairs[i];
            pd.costs = reinterpret_cast<uint8_t*>(data);
            data += pair_cost_bytes((uint32_t)pd.width, (uint32_t)pd.height, specs[i].cfg);
        }

    // Longest work first inside each persistent launch (LPT order): a unit's
    // cost is its longest scanline times D.
    auto unit_cost = [&](const UnitDev& u) -> long long {
        const JobDev& j = pl.jobs[u.job];
        const PairDev& p = pl.pairs[j.pair];
        long long len;
        if (j.dy == 0) len = p.width;
        else if (j.dx == 0) len = p.height;
        else {  // longest of the unit's diagonals
            len = 0;
            const int k0 = j.k_min + u.first_scanline;
            const int per_unit = pl.unit_scanlines == kScanForm ? scan_geometry(p.nd_vec).scanlines
                                                                 : pl.unit_scanlines;
            const int k1 = j.k_min + std::min(u.first_scanline + per_unit, j.num_scanlines);
            for (int k = k0; k < k1; ++k) {
                int tb, te;
                if (j.dx > 0) { tb = std::max(0, -k); te = std::min(p.height, p.width - k); }
                else { tb = std::max(0, k - p.width + 1); te = std::min(p.height, k + 1); }
                len = std::max<long long>(len, te - tb);
            }
        }
        return len * p.nd;
    };
    {
        std::vector<std::pair<long long, int>> order(units.size());
        for (size_t i = 0; i < units.size(); ++i) order[i] = {-unit_cost(units[i]), (int)i};
        std::sort(order.begin(), order.end());
        pl.units.resize(units.size());
        for (size_t i = 0; i < units.size(); ++i) pl.units[i] = units[order[i].second];
    }
    // VX_SGM_AGG_WARPGROUPS=<n> forces the aggregation CTA size of plans that
    // were not given one (the tests run mixed-D batches with several queue
    // classes through it).
    if (warpgroups <= 0)
        if (const char* f = std::getenv("VX_SGM_AGG_WARPGROUPS")) warpgroups = (int)std::strtol(f, nullptr, 10);
    const vx_status qs = plan_queues(pl, warpgroups, unit_cost);
    if (qs != VX_OK) return qs;

    size_t off = 0;
    pl.off_pairs = off;
    off = align_up(off + pl.pairs.size() * sizeof(PairDev));
    pl.off_jobs = off;
    off = align_up(off + pl.jobs.size() * sizeof(JobDev));
    pl.off_units = off;
    off = align_up(off + pl.units.size() * sizeof(UnitDev));
    // Counters: the aggregation work queues, then per pair the escape pool's
    // taken count and overflow flag (all cleared by every launch).
    pl.off_counters = off;
    for (int i = 0; i < n; ++i)
        pl.pairs[i].esc_state = reinterpret_cast<uint32_t*>(pl.off_escape() + sizeof(unsigned) * 2 * (size_t)i);
    off = align_up(off + pl.counter_bytes());
    pl.off_data = off;
    pl.ws_bytes = off + data;
    return VX_OK;
}

void bind_plan(Plan& pl, char* base) {
    char* data = base + pl.off_data;
    for (auto& pd : pl.pairs) {
        pd.census_l = data + reinterpret_cast<size_t>(pd.census_l);
        pd.census_r = data + reinterpret_cast<size_t>(pd.census_r);
        pd.census_lt = data + reinterpret_cast<size_t>(pd.census_lt);
        pd.census_rt = data + reinterpret_cast<size_t>(pd.census_rt);
        pd.slabs = reinterpret_cast<uint8_t*>(data + reinterpret_cast<size_t>(pd.slabs));
        if (pl.unit_scanlines != 32)
            pd.costs = reinterpret_cast<uint8_t*>(data + reinterpret_cast<size_t>(pd.costs));
        pd.shadow = reinterpret_cast<uint16_t*>(data + reinterpret_cast<size_t>(pd.shadow));
        pd.esc_state = reinterpret_cast<uint32_t*>(base + reinterpret_cast<size_t>(pd.esc_state));
    }
}

vx_status upload_plan(const Plan& pl, char* base, cudaStream_t stream, bool pairs_only) {
    const int n = (int)pl.pairs.size();
    if (n == 0) return VX_OK;
    cudaError_t e = cudaMemcpyAsync(base + pl.off_pairs, pl.pairs.data(), n * sizeof(PairDev),
                                    cudaMemcpyHostToDevice, stream);
    if (!pairs_only) {
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(base + pl.off_jobs, pl.jobs.data(), pl.jobs.size() * sizeof(JobDev),
                                cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess && !pl.units.empty())
            e = cudaMemcpyAsync(base + pl.off_units, pl.units.data(),
                                pl.units.size() * sizeof(UnitDev), cudaMemcpyHostToDevice, stream);
    }
    return e == cudaSuccess ? VX_OK : cuda_fail(e, "uploading the batch plan");
}

vx_status launch_plan(const Plan& pl, char* base, cudaStream_t stream, cudaEvent_t* ev, bool capturing) {
    // Under stream capture the timing events become event-record nodes.
    auto record = [&](cudaEvent_t e) {
        if (!e) return;
        if (capturing) cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal);
        else cudaEventRecord(e, stream);
    };
    const int n = (int)pl.pairs.size();
    if (n == 0) return VX_OK;
    cudaError_t e = cudaMemsetAsync(base + pl.off_counters, 0, pl.counter_bytes(), stream);
    if (e != cudaSuccess) return cuda_fail(e, "clearing the work and escape counters");
    const PairDev* d_pairs = reinterpret_cast<const PairDev*>(base + pl.off_pairs);
    const JobDev* d_jobs = reinterpret_cast<const JobDev*>(base + pl.off_jobs);
    const UnitDev* d_units = reinterpret_cast<const UnitDev*>(base + pl.off_units);
    unsigned* counters = reinterpret_cast<unsigned*>(base + pl.off_counters);

    if (ev) record(ev[0]);
    e = launch_census(d_pairs, n, pl.total_tiles, pl.max_rx, pl.max_ry, pl.census64,
                      pl.unit_scanlines == 32, stream);
    if (e != cudaSuccess) return cuda_fail(e, "census launch");
    if (ev) record(ev[1]);
    if (pl.unit_scanlines != 32) {
        e = launch_costs(d_pairs, n, pl.total_rows, pl.dp_max, pl.census64, stream);
        if (e != cudaSuccess) return cuda_fail(e, "cost volume launch");
    }
    if (ev) record(ev[2]);
    e = launch_aggregate(pl.unit_scanlines, pl.dp_max, pl.dp_min, pl.census64, pl.wide_tiles, pl.agg, d_pairs, d_jobs, d_units,
                         (int)pl.units.size(), counters, stream, pl.compact);
    if (e != cudaSuccess) return cuda_fail(e, "aggregation launch");
    if (ev) record(ev[3]);
    e = launch_wta(d_pairs, n, pl.total_rows, pl.max_width, stream);
    if (e != cudaSuccess) return cuda_fail(e, "WTA launch");
    if (ev) record(ev[4]);
    return VX_OK;
}

vx_status run_plan(const Plan& pl, char* base, cudaStream_t stream, cudaEvent_t* ev) {
    vx_status st = upload_plan(pl, base, stream, false);
    if (st != VX_OK) return st;
    return launch_plan(pl, base, stream, ev, false);
}

}  // namespace vxsgm
