// Work-list executor (see hphc_executor.h).
#include "hphc_executor.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "hphc.h"

namespace hphc {
namespace {

constexpr double kInvSqrt2Pi = 0.398942280401432677939946059934;
constexpr double kLog2e = 1.44269504088896340735992468100189214;


size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

double record_scale(double precisionParam) {
    return std::fabs(precisionParam) * std::sqrt(0.5 * kLog2e);
}

// Host replica of the kernel's tile-pair decision (hphc_kernels.cu, tile_mode).
void tile_needs(double tminI, double tmaxI, double tminJ, double tmaxJ, const PairConsts& c,
                bool* doB, bool* doS) {
    const double dtLo = tminI - tmaxJ, dtHi = tmaxI - tminJ;
    const double minAbs = dtLo > 0.0 ? dtLo : (dtHi < 0.0 ? -dtHi : 0.0);
    *doB = !c.noB && !(c.skipB >= 0.0 && -c.cB * minAbs * minAbs >= c.skipB);
    const bool allCausal = dtLo > 0.0;
    *doS = (dtHi > 0.0) && !(c.skipS >= 0.0 && allCausal && -c.cW * dtLo >= c.skipS);
}

// Band [*lo, *hi) of j tiles that strip st (r tiles of targets) must visit:
// every tile that may hold a non-zero term for constants c, plus one tile of
// margin each side; wide: for any sigma and omega (the device-resident
// loop).  For sorted times the tile bounds are non-decreasing, and a tile
// before the strip can hold a background term only if its time gap is below
// dB = sqrt(skipB / -cB), a self-excitation term only below
// dS = skipS / -cW (tile_mode's underflow tests solved for the gap), so each
// edge is one binary search on the bounds.  The band may keep a few tiles
// those tests would drop (tile_mode also tests causality and the space
// coefficient); the sweep decides every tile itself, and chunks sit on a
// fixed grid, so a wider band never changes a bit of the result.
void strip_band(const SetView& s, const PairConsts& c, bool symmetric, bool wide, int r,
                int nTiles, int st, int* loOut, int* hiOut) {
    const int ts0 = st * r, ts1 = std::min(ts0 + r, nTiles);
    *loOut = 0;
    *hiOut = nTiles;
    if (!s.sorted) return;
    const double tminI = s.hTileMin[ts0], tmaxI = s.hTileMax[ts1 - 1];
    // gap beyond which every term of the kind is exactly zero (+inf: none)
    const double kInf = INFINITY;
    const bool anyB = !c.noB;
    const double dB = !anyB ? -kInf
                    : (c.skipB >= 0.0 && c.cB < 0.0 && c.cA <= 0.0) ? std::sqrt(c.skipB / -c.cB)
                                                                      : kInf;
    const double dS = (c.skipS >= 0.0 && c.cW < 0.0 && c.cS <= 0.0) ? c.skipS / -c.cW : kInf;
    // left edge: the first tile before the strip whose gap tminI - tmaxJ is
    // below the larger distance (wide: any sigma, omega, so every tile)
    int lo = 0;
    if (!wide) {
        const double d = std::max(dB, dS);
        if (d < kInf) {
            const double* first = std::upper_bound(s.hTileMax, s.hTileMax + ts0, tminI - d);
            lo = std::max(0, (int)(first - s.hTileMax) - 1);
        }
    }
    // right edge: with the symmetric sweep, later tiles add this strip's
    // pairs as columns (and sorted times leave no self-excitation there);
    // otherwise the first tile after the strip whose gap tminJ - tmaxI is at
    // least dB (background only: no causal pair lies after the strip)
    int hi = ts1;
    if (!symmetric && ts1 < nTiles && dB > -kInf) {
        if (dB == kInf) {
            hi = nTiles;
        } else {
            const double* first = std::lower_bound(s.hTileMin + ts1, s.hTileMin + nTiles,
                                                   tmaxI + dB);
            hi = std::min(nTiles, (int)(first - s.hTileMin) + 1);
        }
    } else if (!symmetric && ts1 < nTiles) {
        hi = std::min(nTiles, ts1 + 1);
    }
    *loOut = lo;
    *hiOut = hi;
}

// Relative cost of the tiles of one work item, for ordering the work list
// (largest first) and dealing strips to ranks.  For sorted times a strip's
// tiles split by their time gap to the strip: below dF = sqrt(fastB / -cB)
// the background terms take the full exponential ("near"), beyond it the
// far tail's cheaper one; below dS the tile also holds self-excitation
// terms.  Weights from measured sweep times: a far-tail tile costs about
// half a near one in the FP32-compensated mode (whose near terms take the
// software exponential and three compensated sums) and 7/10 in the FP64
// mode; the self-excitation terms of a tile add about half a tile in the
// FP32 mode and a whole one in the FP64 mode (CUDA's exp() for each).
// Ordering by these costs instead of tile counts: sweep at N = 100k 2.588 ->
// 2.498 ms (FP32, plain block sums then) and 10.06 -> 9.69 ms (FP64); the
// FP32 far weight 0.75 -> 0.5 with the compensated sums: 2.676 -> 2.620 ms
// at 64 items/SM, 2.81 -> 2.64 ms at 32.
constexpr double kFarTileCostF32 = 0.5;
constexpr double kFarTileCostF64 = 0.70;
constexpr double kSelfTileCostF32 = 0.5;
constexpr double kSelfTileCostF64 = 1.0;

struct StripCost {
    int nearLo = 0, nearHi = 0;  // near background tiles
    int selfLo = 0, selfHi = 0;  // tiles with self-excitation terms
    double far = 1.0;            // weight of a background tile outside [nearLo, nearHi)
    double self = kSelfTileCostF32;  // added weight of a tile with self-excitation terms
};

StripCost strip_cost(const SetView& s, const PairConsts& c, bool fp32, int r, int nTiles,
                     int st) {
    StripCost k;
    k.self = fp32 ? kSelfTileCostF32 : kSelfTileCostF64;
    const int ts0 = st * r, ts1 = std::min(ts0 + r, nTiles);
    k.nearLo = 0;
    k.nearHi = nTiles;
    k.selfLo = 0;
    k.selfHi = ts1;
    if (!s.sorted) return k;
    const double tminI = s.hTileMin[ts0], tmaxI = s.hTileMax[ts1 - 1];
    if (c.fastB > 0.0 && c.cB < 0.0 && c.cA <= 0.0) {
        const double dF = std::sqrt(c.fastB / -c.cB);
        k.nearLo = (int)(std::upper_bound(s.hTileMax, s.hTileMax + ts0, tminI - dF) - s.hTileMax);
        k.nearHi = (int)(std::lower_bound(s.hTileMin + ts1, s.hTileMin + nTiles, tmaxI + dF) -
                         s.hTileMin);
        k.far = fp32 ? kFarTileCostF32 : kFarTileCostF64;
    }
    if (c.skipS >= 0.0 && c.cW < 0.0 && c.cS <= 0.0) {
        const double dS = c.skipS / -c.cW;
        k.selfLo = (int)(std::upper_bound(s.hTileMax, s.hTileMax + ts0, tminI - dS) - s.hTileMax);
    }
    return k;
}

double item_cost(const StripCost& k, bool noB, int jt0, int jt1) {
    const auto overlap = [&](int a, int b) { return std::max(0, std::min(jt1, b) - std::max(jt0, a)); };
    const int near = overlap(k.nearLo, k.nearHi);
    const double b = noB ? 0.0 : near + k.far * (jt1 - jt0 - near);
    return b + k.self * overlap(k.selfLo, k.selfHi);
}

int f32_stride(int D) {
    return (2 * (D + 1) + 1 + 3) / 4 * 4;
}

// Autotuned sweep shapes per process: (D, precision, mode bits, log2 of the
// pair count, log2 of the problem count) -> (R, items per SM).
using TuneKey = std::tuple<int, int, int, int, int>;
std::mutex gTuneMutex;
std::map<TuneKey, std::pair<int, int>> gTuneCache;

// Persistent tune cache: HPHC_TUNE_CACHE names a file of JSON lines, one per
// tuned shape,
//   {"v":1,"device":"<name>","sms":148,"D":2,"precision":1,"mode":50,
//    "pairs_log2":34,"problems_log2":0,"R":4,"items":64}
// read once per process (lines of other devices, other versions or with an
// invalid shape are ignored) and appended to after each new tuning.  Each
// line is written with one append of under 200 bytes, so processes sharing
// the file do not interleave their lines.
constexpr int kTuneCacheVersion = 1;
constexpr int kTuneReps = 4;  // timed sweeps per candidate shape (even)

struct TuneLine {
    std::string device;
    int sms;
    TuneKey key;
    int R, items;
};
std::vector<TuneLine> gTuneFile;
bool gTuneFileRead = false;

// Position of the value of "key" in a one-line JSON object (after the
// colon and any blanks), or npos.
size_t json_value(const std::string& line, const char* key) {
    const std::string k = std::string("\"") + key + "\"";
    size_t at = line.find(k);
    if (at == std::string::npos) return at;
    at = line.find_first_not_of(" \t", at + k.size());
    if (at == std::string::npos || line[at] != ':') return std::string::npos;
    return line.find_first_not_of(" \t", at + 1);
}

bool json_int(const std::string& line, const char* key, int* out) {
    const size_t at = json_value(line, key);
    if (at == std::string::npos) return false;
    char* end = nullptr;
    const long v = std::strtol(line.c_str() + at, &end, 10);
    if (end == line.c_str() + at) return false;
    *out = (int)v;
    return true;
}

bool json_string(const std::string& line, const char* key, std::string* out) {
    const size_t at = json_value(line, key);
    if (at == std::string::npos || line[at] != '"') return false;
    const size_t end = line.find('"', at + 1);
    if (end == std::string::npos) return false;
    *out = line.substr(at + 1, end - at - 1);
    return true;
}

bool valid_shape(int precision, int R, int items) {
    const bool okR = precision == HPHC_PRECISION_FP64 ? (R == 1 || R == 2) : (R == 2 || R == 4);
    return okR && items >= 1 && items <= 1024;
}

// Called with gTuneMutex held.
void read_tune_file() {
    if (gTuneFileRead) return;
    gTuneFileRead = true;
    const char* path = std::getenv("HPHC_TUNE_CACHE");
    if (!path || !*path) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char buf[512];
    while (std::fgets(buf, sizeof buf, f)) {
        const std::string line(buf);
        TuneLine t;
        int v = 0, D = 0, prec = 0, mode = 0, pb = 0, kb = 0;
        if (!json_int(line, "v", &v) || v != kTuneCacheVersion) continue;
        if (!json_string(line, "device", &t.device) || !json_int(line, "sms", &t.sms) ||
            !json_int(line, "D", &D) || !json_int(line, "precision", &prec) ||
            !json_int(line, "mode", &mode) || !json_int(line, "pairs_log2", &pb) ||
            !json_int(line, "problems_log2", &kb) || !json_int(line, "R", &t.R) ||
            !json_int(line, "items", &t.items))
            continue;
        if (!valid_shape(prec, t.R, t.items)) continue;
        t.key = std::make_tuple(D, prec, mode, pb, kb);
        gTuneFile.push_back(t);
    }
    std::fclose(f);
}

void append_tune_file(const std::string& device, int sms, const TuneKey& key, int R, int items) {
    const char* path = std::getenv("HPHC_TUNE_CACHE");
    if (!path || !*path) return;
    std::string name = device;
    for (char& ch : name)
        if (ch == '"' || ch == '\\' || (unsigned char)ch < 0x20) ch = '_';
    char line[400];
    const int n = std::snprintf(
        line, sizeof line,
        "{\"v\":%d,\"device\":\"%s\",\"sms\":%d,\"D\":%d,\"precision\":%d,\"mode\":%d,"
        "\"pairs_log2\":%d,\"problems_log2\":%d,\"R\":%d,\"items\":%d}\n",
        kTuneCacheVersion, name.c_str(), sms, std::get<0>(key), std::get<1>(key),
        std::get<2>(key), std::get<3>(key), std::get<4>(key), R, items);
    if (n <= 0 || n >= (int)sizeof line) return;
    FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fwrite(line, 1, (size_t)n, f);
    std::fclose(f);
}

int log2_bucket(double x) {
    int b = 0;
    while (x > 1.0 && b < 80) {
        x *= 0.5;
        ++b;
    }
    return b;
}

}  // namespace

int Executor::cuda_fail(cudaError_t e, const char* what) {
    error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? HPHC_ERR_OUT_OF_MEMORY : HPHC_ERR_CUDA;
}

int Executor::init(int D, int precision, int variant, bool underflowSkip, int device,
                   cudaStream_t stream, double ex2Bias) {
    D_ = D;
    precision_ = precision;
    variant_ = variant;
    skip_ = underflowSkip;
    device_ = device;
    stream_ = stream;
    ex2Bias_ = ex2Bias;
    cudaDeviceGetAttribute(&numSMs_, cudaDevAttrMultiProcessorCount, device);
    R = precision == HPHC_PRECISION_FP64 ? 2 : 4;
    itemsPerSM = 32;
    cudaError_t e = cudaMalloc(&dCounter_, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "device allocation");
    for (auto& ev : ev_)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return cuda_fail(e, "create events");
    return HPHC_OK;
}

void Executor::drop_graph() {
    if (graphExec_) cudaGraphExecDestroy(graphExec_);
    graphExec_ = nullptr;
    graphKey_ = GraphKey{};
}

void Executor::release() {
    drop_graph();
    if (dTables_) cudaFree(dTables_);
    if (hStaging_) cudaFreeHost(hStaging_);
    if (dRecPool_) cudaFree(dRecPool_);
    if (dPartials_) cudaFree(dPartials_);
    if (dColAcc_) cudaFree(dColAcc_);
    if (dBlockSums_) cudaFree(dBlockSums_);
    if (dOut_) cudaFree(dOut_);
    if (hOut_) cudaFreeHost(hOut_);
    if (dCounter_) cudaFree(dCounter_);
    for (auto& ev : ev_)
        if (ev) cudaEventDestroy(ev);
    dTables_ = hStaging_ = nullptr;
    dRecPool_ = nullptr;
    dPartials_ = dBlockSums_ = dOut_ = hOut_ = nullptr;
    dColAcc_ = nullptr;
    dCounter_ = nullptr;
    tablesCap_ = stagingCap_ = recCap_ = partialsCap_ = blockCap_ = outCap_ = colCap_ = 0;
    for (auto& ev : ev_) ev = nullptr;
}

ConstsSpec Executor::consts_spec() const {
    ConstsSpec s{};
    s.precision = precision_ == HPHC_PRECISION_FP64 ? 0 : 1;
    s.D = D_;
    s.variant = variant_;
    s.skip = skip_ ? 1 : 0;
    s.truncate = (skip_ && truncateTail) ? 1 : 0;
    s.ex2Bias = ex2Bias_;
    s.fastTail = fastTail ? 1 : 0;
    s.noB = keptB ? 1 : 0;
    return s;
}

PairConsts Executor::pair_consts(const double* p) const {
    PairConsts c{};
    FinishConsts f{};
    param_consts(p, consts_spec(), c, f);
    return c;
}

FinishConsts Executor::finish_consts(const double* p, const SetView& set) const {
    PairConsts c{};
    FinishConsts f{};
    param_consts(p, consts_spec(), c, f);
    f.T = set.hTimes[set.N - 1];
    // src/NewHawkes.hpp:659: locationCount * (embeddingDimension - 1) * log(M_1_SQRT_2PI)
    f.constant = (double)(set.N * (D_ - 1)) * std::log(kInvSqrt2Pi);
    return f;
}

int Executor::sweep_grid(int r) const {
    const int perSM = sweep_list_blocks_per_sm(precision_ == HPHC_PRECISION_FP64 ? 0 : 1, D_, r,
                                               variant_);
    return numSMs_ * std::max(1, perSM);
}

int Executor::build_plan(const std::vector<SetView>& sets, const int* setOf, const double* params,
                         int P, double* dProbs, int r, int items) {
    Plan& pl = plan_;
    pl.P = P;
    pl.setOf.assign(setOf, setOf + P);
    pl.sp.assign(P, SweepProblem{});
    pl.fp.assign(P, FinishProblem{});
    pl.pj.clear();
    pl.items.clear();
    pl.stripChunks.clear();
    pl.fb.clear();
    pl.maxN = 0;
    const bool fp32 = precision_ != HPHC_PRECISION_FP64;
    const int stripEvents = kSweepThreads * r;
    const int S32 = f32_stride(D_);

    double totalStrips = 0.0;
    for (int p = 0; p < P; ++p) {
        const SetView& s = sets[setOf[p]];
        totalStrips += (s.N + stripEvents - 1) / stripEvents;
    }
    // a shard keeps about 1/shardWorld of the items: cut finer chunks so that
    // each rank still has `items` per SM
    const int target = numSMs_ * items * std::max(1, shardWorld);
    const int nChunksTarget = std::max(1, (int)std::ceil(target / std::max(1.0, totalStrips)));

    // A self-excitation-only sweep (kept background sums, host-planned bands)
    // visits a few tiles near each strip.  With fewer strips than two per
    // resident CTA (one problem, say), the general grid leaves about one wave
    // of items, where the few left over double the sweep's time: the bands
    // are then cut on a grid set from their total, estimated from up to 16
    // strips a problem, for about four items per resident CTA (never coarser
    // than the general grid).  With more strips each band stays one item.
    int selfCT = 0;
    if (keptB && !wideBands_ && totalStrips < 2.0 * sweep_grid(r)) {
        double bandTiles = 0.0;
        for (int p = 0; p < P; ++p) {
            const SetView& s = sets[setOf[p]];
            const PairConsts c = pair_consts(params + (size_t)6 * p);
            const int nTiles = (s.N + kTile - 1) / kTile;
            const int nStrips = (s.N + stripEvents - 1) / stripEvents;
            const int step = std::max(1, nStrips / 16);
            double sampled = 0.0;
            int n = 0;
            for (int st = 0; st < nStrips; st += step, ++n) {
                int lo = 0, hi = nTiles;
                strip_band(s, c, false, false, r, nTiles, st, &lo, &hi);
                sampled += hi - lo;
            }
            bandTiles += sampled * nStrips / std::max(1, n);
        }
        // a power of two near it, so that small changes of the bands (a
        // sampler's steps in omega) keep the grid, the list's capacity and
        // the captured graph
        const double want = std::max(1.0, bandTiles / (4.0 * sweep_grid(r)));
        selfCT = 1 << (int)std::lround(std::log2(want));
    }

    size_t recOff = 0, partOff = 0, colOff = 0;
    std::vector<size_t> chunkBase(P);
    std::vector<double> itemCost;  // parallel to pl.items
    int blockBase = 0;
    for (int p = 0; p < P; ++p) {
        const SetView& s = sets[setOf[p]];
        const double* prm = params + (size_t)6 * p;
        if (fp32 && !(prm[1] != 0.0 && prm[2] != 0.0 && std::isfinite(prm[1]) &&
                      std::isfinite(prm[2]))) {
            char buf[200];
            snprintf(buf, sizeof buf,
                     "FP32-compensated mode needs finite non-zero tauXprec and tauTprec (problem "
                     "%d: %g, %g); use the FP64 mode", p, prm[1], prm[2]);
            error = buf;
            return HPHC_ERR_UNSUPPORTED;
        }
        const int N = s.N;
        const int nTiles = (N + kTile - 1) / kTile;
        const int nStrips = (N + stripEvents - 1) / stripEvents;
        const int Npad = nStrips * stripEvents;
        // tiles a chunk (a self-excitation-only grid never coarser than the
        // general one, which follows the tuned items per SM)
        const int generalCT = std::max(1, (nTiles + nChunksTarget - 1) / nChunksTarget);
        const int CT = selfCT > 0 ? std::min(selfCT, generalCT) : generalCT;
        int maxSlots = 1;  // partial-sum slots the widest strip band uses
        pl.maxN = std::max(pl.maxN, N);
        SweepProblem& sp = pl.sp[p];
        sp.c = pair_consts(prm);
        sp.N = N;
        sp.nTiles = nTiles;
        sp.Npad = Npad;
        sp.tileMin = s.dTileMin;
        sp.tileMax = s.dTileMax;
        // a self-excitation-only sweep has no background, so no column sums
        sp.symmetric = (symmetric && !keptB && N <= kMaxSymmetricEvents) ? 1 : 0;
        if (!fp32 && sp.symmetric) {
            // FP64 column sums are fixed point: bound each column total by N
            // times the largest term, B_u <= 1, B_u d^2 <= 1/(e |cA|),
            // B_u dt^2 <= 1/(e |cB|), and keep it below 2^62 units.  Padding
            // rows 1e150 away vanish only if |cA| is not astronomically small.
            if (!(sp.c.cA < -1e-280 && sp.c.cB < 0.0)) {
                sp.symmetric = 0;
            } else {
                const double e1 = std::exp(1.0);
                const double bound[3] = {(double)N, N / (e1 * -sp.c.cA), N / (e1 * -sp.c.cB)};
                for (int q = 0; q < 3; ++q) {
                    int ex = 0;
                    std::frexp(bound[q], &ex);  // bound < 2^ex
                    sp.colShift[q] = 62 - ex;
                }
            }
        }
        sp.searchBand = (wideBands_ && s.sorted) ? 1 : 0;
        sp.rowOrder = (fp32 && sp.symmetric) ? (r == 2 ? s.dOrder2 : r == 4 ? s.dOrder4 : nullptr)
                                             : nullptr;
        sp.colAcc = nullptr;
        if (sp.symmetric) {
            sp.colAcc = reinterpret_cast<unsigned long long*>(colOff + 1);  // offset + 1
            colOff += (size_t)(fp32 ? 3 : 6) * Npad;
        }
        if (fp32) {
            // problems on the same set with the same tauX and tauT (sampler
            // chains, proposals that leave them fixed) share one record copy
            const double sX = record_scale(prm[1]), sT = record_scale(prm[2]);
            size_t off = recOff;
            bool shared = false;
            for (const PackJob& j : pl.pj)
                if (j.loc == s.dLoc && j.sX == sX && j.sT == sT) {
                    off = reinterpret_cast<size_t>(j.rec);
                    shared = true;
                    break;
                }
            sp.rec = reinterpret_cast<const void*>(off);  // offset, fixed up later
            if (!shared) {
                PackJob j{};
                j.loc = s.dLoc;
                j.times = s.dTimes;
                j.ranks = s.dRanks;
                j.rec = reinterpret_cast<float*>(recOff);
                j.sX = sX;
                j.sT = sT;
                j.N = N;
                pl.pj.push_back(j);
                recOff += (size_t)N * S32;
            }
        } else {
            sp.rec = s.dRecF64;
        }

        // work items: each strip's band of tiles that may hold a non-zero term
        chunkBase[p] = pl.stripChunks.size();
        for (int st = 0; st < nStrips; ++st) {
            int lo = 0, hi = nTiles;
            strip_band(s, sp.c, sp.symmetric != 0, wideBands_, r, nTiles, st, &lo, &hi);
            const StripCost sc = strip_cost(s, sp.c, fp32, r, nTiles, st);
            // Chunks sit on a fixed grid of CT tiles per problem, so a tile
            // always lands in the same chunk whatever the band: skipping a
            // band's outside only drops chunks whose sums are exactly zero,
            // and the FP64 chunk sums are added in the same order either way.
            const int cFirst = lo / CT, cLast = (hi - 1) / CT + 1;
            for (int c = cFirst; c < cLast; ++c) {
                WorkItem w{};
                w.problem = p;
                w.strip = st;
                w.jt0 = std::max(lo, c * CT);
                w.jt1 = std::min(hi, (c + 1) * CT);
                w.slot = c - cFirst;
                w.start = w.jt0;
                pl.items.push_back(w);
                itemCost.push_back(item_cost(sc, sp.c.noB != 0, w.jt0, w.jt1));
            }
            pl.stripChunks.push_back(cLast - cFirst);
            maxSlots = std::max(maxSlots, cLast - cFirst);
        }
        // partial sums: as many slots per strip as the widest band uses
        sp.partials = reinterpret_cast<double*>(partOff);  // offset, fixed up later
        partOff += (size_t)maxSlots * kNumAcc * Npad;

        FinishProblem& fp = pl.fp[p];
        fp.partials = nullptr;  // fixed up later
        fp.colAcc = nullptr;
        fp.stripChunks = nullptr;
        fp.times = s.dTimes;
        fp.probs = (p == 0) ? dProbs : nullptr;
        fp.sums = (p == 0) ? sumsOut : nullptr;
        fp.keptB = keptB;
        fp.N = N;
        fp.Npad = Npad;
        fp.stripEvents = stripEvents;
        fp.blockBase = blockBase;
        fp.nBlocks = finish_blocks(N);
        fp.colWords = fp32 ? 1 : 2;
        for (int q = 0; q < 4; ++q) fp.colShift[q] = sp.colShift[q];
        fp.f = finish_consts(prm, s);
        for (int b = 0; b < fp.nBlocks; ++b) pl.fb.push_back(FinishBlock{p, b * kFinishThreads});
        blockBase += fp.nBlocks;
    }
    pl.nBlocks = blockBase;
    if (shardWorld > 1) {
        // Longest-processing-time assignment of whole strips to ranks by
        // their item costs; ties go to the lower strip and the lower rank,
        // so every rank derives the same assignment from the same plan.
        const size_t nS = pl.stripChunks.size();
        std::vector<double> cost(nS, 0.0);
        for (size_t k = 0; k < pl.items.size(); ++k)
            cost[chunkBase[pl.items[k].problem] + pl.items[k].strip] += itemCost[k];
        std::vector<int> order(nS);
        for (size_t k = 0; k < nS; ++k) order[k] = (int)k;
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return cost[x] > cost[y]; });
        std::vector<double> load(shardWorld, 0.0);
        std::vector<char> owned(nS, 0);
        for (int k : order) {
            int best = 0;
            for (int r = 1; r < shardWorld; ++r)
                if (load[r] < load[best]) best = r;
            load[best] += cost[k];
            owned[k] = best == shardRank;
        }
        size_t kept = 0;
        for (size_t k = 0; k < pl.items.size(); ++k)
            if (owned[chunkBase[pl.items[k].problem] + pl.items[k].strip]) {
                itemCost[kept] = itemCost[k];
                pl.items[kept++] = pl.items[k];
            }
        pl.items.resize(kept);
        itemCost.resize(kept);
        for (size_t k = 0; k < nS; ++k)
            if (!owned[k]) pl.stripChunks[k] = 0;
    }
    // largest first, so that the persistent CTAs end on small items
    {
        std::vector<int> order(pl.items.size());
        for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return itemCost[x] > itemCost[y]; });
        std::vector<WorkItem> sorted(order.size());
        for (size_t k = 0; k < order.size(); ++k) sorted[k] = pl.items[order[k]];
        pl.items.swap(sorted);
    }

    // table layout and buffer capacities
    offSP_ = 0;
    offItems_ = align16(offSP_ + sizeof(SweepProblem) * P);
    const size_t nItems = pl.items.size();
    itemsCap_ = std::max(itemsCap_, nItems);
    offNItems_ = align16(offItems_ + sizeof(WorkItem) * itemsCap_);
    offChunks_ = align16(offNItems_ + sizeof(int));
    offFP_ = align16(offChunks_ + sizeof(int) * pl.stripChunks.size());
    offFB_ = align16(offFP_ + sizeof(FinishProblem) * P);
    offPJ_ = align16(offFB_ + sizeof(FinishBlock) * pl.fb.size());
    tablesBytes_ = align16(offPJ_ + sizeof(PackJob) * pl.pj.size());

    recNeed_ = recOff;
    partialsNeed_ = partOff;
    colNeed_ = colOff;
    int st = ensure_buffers();
    if (st) return st;

    // fix up offsets into device pointers and fill the staging buffer
    char* h = static_cast<char*>(hStaging_);
    char* d = static_cast<char*>(dTables_);
    for (int p = 0; p < P; ++p) {
        SweepProblem& sp = pl.sp[p];
        const size_t po = reinterpret_cast<size_t>(sp.partials);
        sp.partials = dPartials_ + po;
        if (sp.colAcc) sp.colAcc = dColAcc_ + (reinterpret_cast<size_t>(sp.colAcc) - 1);
        if (fp32) sp.rec = dRecPool_ + reinterpret_cast<size_t>(sp.rec);
        FinishProblem& fp = pl.fp[p];
        fp.partials = sp.partials;
        fp.colAcc = sp.colAcc;
        fp.stripChunks = reinterpret_cast<const int*>(d + offChunks_) + chunkBase[p];
    }
    for (auto& j : pl.pj) j.rec = dRecPool_ + reinterpret_cast<size_t>(j.rec);
    std::memcpy(h + offSP_, pl.sp.data(), sizeof(SweepProblem) * P);
    std::memcpy(h + offItems_, pl.items.data(), sizeof(WorkItem) * nItems);
    const int n = (int)nItems;
    std::memcpy(h + offNItems_, &n, sizeof(int));
    std::memcpy(h + offChunks_, pl.stripChunks.data(), sizeof(int) * pl.stripChunks.size());
    std::memcpy(h + offFP_, pl.fp.data(), sizeof(FinishProblem) * P);
    std::memcpy(h + offFB_, pl.fb.data(), sizeof(FinishBlock) * pl.fb.size());
    if (!pl.pj.empty()) std::memcpy(h + offPJ_, pl.pj.data(), sizeof(PackJob) * pl.pj.size());
    return HPHC_OK;
}

int Executor::ensure_buffers() {
    const Plan& pl = plan_;
    bool grew = false;
    cudaError_t e = cudaSuccess;
    auto grow_dev = [&](void** ptr, size_t& cap, size_t needBytes) -> cudaError_t {
        if (needBytes <= cap && *ptr) return cudaSuccess;
        const size_t n = std::max<size_t>(needBytes + needBytes / 4, 256);
        if (*ptr) cudaFree(*ptr);
        *ptr = nullptr;
        cap = 0;
        const cudaError_t err = cudaMalloc(ptr, n);
        if (err == cudaSuccess) cap = n;
        grew = true;
        return err;
    };
    if ((e = grow_dev(reinterpret_cast<void**>(&dRecPool_), recCap_,
                      std::max<size_t>(recNeed_, 1) * sizeof(float))) != cudaSuccess ||
        (e = grow_dev(reinterpret_cast<void**>(&dPartials_), partialsCap_,
                      std::max<size_t>(partialsNeed_, 1) * sizeof(double))) != cudaSuccess ||
        (e = grow_dev(reinterpret_cast<void**>(&dColAcc_), colCap_,
                      std::max<size_t>(colNeed_, 1) * sizeof(unsigned long long))) !=
            cudaSuccess ||
        (e = grow_dev(reinterpret_cast<void**>(&dBlockSums_), blockCap_,
                      (size_t)std::max(pl.nBlocks, 1) * 8 * sizeof(double))) != cudaSuccess ||
        (e = grow_dev(&dTables_, tablesCap_, tablesBytes_)) != cudaSuccess)
        return cuda_fail(e, "device allocation");
    if (stagingCap_ < tablesCap_) {
        if (hStaging_) cudaFreeHost(hStaging_);
        hStaging_ = nullptr;
        stagingCap_ = 0;
        if ((e = cudaMallocHost(&hStaging_, tablesCap_)) != cudaSuccess)
            return cuda_fail(e, "pinned allocation");
        stagingCap_ = tablesCap_;
        grew = true;
    }
    if (outCap_ < (size_t)pl.P * 8) {
        if (dOut_) cudaFree(dOut_);
        if (hOut_) cudaFreeHost(hOut_);
        dOut_ = hOut_ = nullptr;
        outCap_ = 0;
        const size_t n = (size_t)pl.P * 8;
        if ((e = cudaMalloc(&dOut_, n * sizeof(double))) != cudaSuccess ||
            (e = cudaMallocHost(&hOut_, n * sizeof(double))) != cudaSuccess)
            return cuda_fail(e, "device allocation");
        outCap_ = n;
        grew = true;
    }
    if (grew) drop_graph();
    return HPHC_OK;
}

// Timing events: inside a stream capture an event is only recorded as a graph
// node (and so usable for elapsed times) when marked external.
cudaError_t Executor::record(cudaEvent_t ev) {
    return capturing_ ? cudaEventRecordWithFlags(ev, stream_, cudaEventRecordExternal)
                      : cudaEventRecord(ev, stream_);
}

// The stage sequence of one run on stream_ (also what the graph captures).
int Executor::launch_sequence(int grid) {
    const Plan& pl = plan_;
    const int prec = precision_ == HPHC_PRECISION_FP64 ? 0 : 1;
    char* d = static_cast<char*>(dTables_);
    const auto* sp = reinterpret_cast<const SweepProblem*>(d + offSP_);
    const auto* items = reinterpret_cast<const WorkItem*>(d + offItems_);
    const auto* nItems = reinterpret_cast<const int*>(d + offNItems_);
    const auto* fp = reinterpret_cast<const FinishProblem*>(d + offFP_);
    const auto* fb = reinterpret_cast<const FinishBlock*>(d + offFB_);
    const auto* pj = reinterpret_cast<const PackJob*>(d + offPJ_);
    cudaError_t e = cudaSuccess;
    int launches = 0;
    if (kernelTiming && (e = record(ev_[0]))) return cuda_fail(e, "timing event");
    if ((e = cudaMemcpyAsync(dTables_, hStaging_, tablesBytes_, cudaMemcpyHostToDevice, stream_)))
        return cuda_fail(e, "stage tables");
    if (prec == 1) {
        if ((e = launch_pack_f32_jobs(D_, (int)pl.pj.size(), pl.maxN, pj, stream_)))
            return cuda_fail(e, "pack kernel");
        ++launches;
    }
    if ((e = cudaMemsetAsync(dCounter_, 0, sizeof(int), stream_)))
        return cuda_fail(e, "reset work counter");
    if (colNeed_ && (e = cudaMemsetAsync(dColAcc_, 0, colNeed_ * sizeof(unsigned long long),
                                         stream_)))
        return cuda_fail(e, "reset column sums");
    if (kernelTiming && (e = record(ev_[1]))) return cuda_fail(e, "timing event");
    if ((e = launch_sweep_list(prec, D_, R, variant_, grid, sp, items, nItems, dCounter_, stream_)))
        return cuda_fail(e, "sweep kernel");
    if (kernelTiming && (e = record(ev_[2]))) return cuda_fail(e, "timing event");
    if ((e = launch_finish_list(pl.nBlocks, fp, fb, dBlockSums_, stream_)))
        return cuda_fail(e, "finish kernel");
    if ((e = launch_final_list(pl.P, fp, dBlockSums_, dOut_, stream_)))
        return cuda_fail(e, "final kernel");
    launches += 3;
    if ((e = cudaMemcpyAsync(hOut_, dOut_, (size_t)pl.P * 8 * sizeof(double),
                             cudaMemcpyDeviceToHost, stream_)))
        return cuda_fail(e, "read results");
    if (kernelTiming && (e = record(ev_[3]))) return cuda_fail(e, "timing event");
    lastLaunches = launches;
    return HPHC_OK;
}

int Executor::autotune(const std::vector<SetView>& sets, const int* setOf, const double* params,
                       int P, double* dProbs) {
    double pairs = 0.0;
    for (int p = 0; p < P; ++p) pairs += (double)sets[setOf[p]].N * sets[setOf[p]].N;
    pairs /= std::max(1, shardWorld);  // work of this rank
    const int mode = variant_ | (symmetric ? 16 : 0) | (fastTail ? 32 : 0) | (skip_ ? 64 : 0) |
                     (truncateTail ? 128 : 0);
    const TuneKey key = std::make_tuple(D_, precision_, mode, log2_bucket(pairs), log2_bucket(P));
    if (deviceName_.empty()) {
        cudaDeviceProp prop{};
        deviceName_ = cudaGetDeviceProperties(&prop, device_) == cudaSuccess ? prop.name : "?";
    }
    {
        std::lock_guard<std::mutex> lock(gTuneMutex);
        auto it = gTuneCache.find(key);
        if (it == gTuneCache.end()) {
            read_tune_file();
            for (const TuneLine& t : gTuneFile)
                if (t.key == key && t.sms == numSMs_ && t.device == deviceName_) {
                    it = gTuneCache.emplace(key, std::make_pair(t.R, t.items)).first;
                    break;
                }
        }
        if (it != gTuneCache.end()) {
            R = fixedR ? fixedR : it->second.first;
            itemsPerSM = fixedItems ? fixedItems : it->second.second;
            tuned_ = true;
            return HPHC_OK;
        }
    }
    std::vector<int> rs, its;
    if (fixedR) rs = {fixedR};
    else if (precision_ == HPHC_PRECISION_FP64) rs = {1, 2};
    else rs = {2, 4};
    if (fixedItems) its = {fixedItems};
    else its = {8, 16, 32, 64};
    const bool timing = kernelTiming;
    kernelTiming = true;
    float best = 1e30f;
    int bestR = rs[0], bestI = its[0];
    int st = HPHC_OK;
    for (int r : rs) {
        for (int it : its) {
            R = r;
            itemsPerSM = it;
            if ((st = build_plan(sets, setOf, params, P, dProbs, r, it))) break;
            const int grid = sweep_grid(r);
            // median of four sweeps after one that warms the caches: the
            // shapes' typical times differ by ~1 %, about as much as the
            // best of a few launches varies
            float times[kTuneReps];
            int nt = 0;
            for (int rep = 0; rep <= kTuneReps && !st; ++rep) {
                if ((st = launch_sequence(grid))) break;
                cudaError_t e = cudaStreamSynchronize(stream_);
                float t = 0.f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ev_[1], ev_[2]);
                if (e != cudaSuccess) {
                    st = cuda_fail(e, "autotune timing");
                    break;
                }
                if (rep > 0) times[nt++] = t;
            }
            float ms = 1e30f;
            if (!st && nt == kTuneReps) {
                std::sort(times, times + nt);
                ms = 0.5f * (times[nt / 2 - 1] + times[nt / 2]);
            }
            if (st) break;
            if (ms < best) {
                best = ms;
                bestR = r;
                bestI = it;
            }
        }
        if (st) break;
    }
    kernelTiming = timing;
    if (st) return st;
    if (!fixedR && !fixedItems) {  // a shape tuned under a constraint is not cached
        std::lock_guard<std::mutex> lock(gTuneMutex);
        gTuneCache[key] = {bestR, bestI};
        append_tune_file(deviceName_, numSMs_, key, bestR, bestI);
    }
    R = bestR;
    itemsPerSM = bestI;
    tuned_ = true;
    return HPHC_OK;
}

int Executor::enqueue(const std::vector<SetView>& sets, const int* setOf, const double* params,
                      int P, double* dProbs) {
    if (P < 1) {
        error = "no problems to evaluate";
        return HPHC_ERR_BAD_ARGUMENT;
    }
    if (fixedR && fixedItems) {
        R = fixedR;
        itemsPerSM = fixedItems;
        tuned_ = true;
    }
    if (!tuned_) {
        const int st = autotune(sets, setOf, params, P, dProbs);
        if (st) return st;
    }
    int st = build_plan(sets, setOf, params, P, dProbs, R, itemsPerSM);
    if (st) return st;
    const int grid = sweep_grid(R);
    timedValid = false;
    if (!useGraph) {
        st = launch_sequence(grid);
        timedValid = kernelTiming && st == HPHC_OK;
        return st;
    }
    GraphKey key;
    key.P = plan_.P;
    key.nJobs = (int)plan_.pj.size();
    key.nBlocks = plan_.nBlocks;
    key.maxN = plan_.maxN;
    key.R = R;
    key.grid = grid;
    key.tablesBytes = tablesBytes_;
    key.colNeed = colNeed_;
    key.tables = dTables_;
    key.timing = kernelTiming;
    const bool same = graphExec_ && key.P == graphKey_.P && key.nJobs == graphKey_.nJobs &&
                      key.nBlocks == graphKey_.nBlocks &&
                      key.maxN == graphKey_.maxN && key.R == graphKey_.R &&
                      key.grid == graphKey_.grid && key.tablesBytes == graphKey_.tablesBytes &&
                      key.colNeed == graphKey_.colNeed &&
                      key.tables == graphKey_.tables && key.timing == graphKey_.timing;
    cudaError_t e;
    if (!same) {
        drop_graph();
        cudaGraph_t graph = nullptr;
        if ((e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal)))
            return cuda_fail(e, "begin graph capture");
        capturing_ = true;
        st = launch_sequence(grid);
        capturing_ = false;
        e = cudaStreamEndCapture(stream_, &graph);
        if (st) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "end graph capture");
        e = cudaGraphInstantiate(&graphExec_, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            graphExec_ = nullptr;
            return cuda_fail(e, "instantiate graph");
        }
        graphKey_ = key;
    }
    if (take_fault(HPHC_FAULT_LAUNCH))
        return cuda_fail(cudaErrorLaunchOutOfResources, "launch graph (injected)");
    if ((e = cudaGraphLaunch(graphExec_, stream_))) return cuda_fail(e, "launch graph");
    lastLaunches = (precision_ == HPHC_PRECISION_FP64 ? 3 : 4);
    timedValid = kernelTiming;
    return HPHC_OK;
}

int Executor::wait(double* hostOut) {
    const cudaError_t e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) return cuda_fail(e, "evaluation");
    if (take_fault(HPHC_FAULT_WAIT)) {
        timedValid = false;
        return cuda_fail(cudaErrorLaunchTimeout, "evaluation (injected)");
    }
    if (hostOut) std::memcpy(hostOut, hOut_, (size_t)plan_.P * 8 * sizeof(double));
    if (timedValid) {
        cudaError_t t;
        if ((t = cudaEventElapsedTime(&lastSweepMs, ev_[1], ev_[2])) != cudaSuccess ||
            (t = cudaEventElapsedTime(&lastFinishMs, ev_[2], ev_[3])) != cudaSuccess ||
            (t = cudaEventElapsedTime(&lastStepMs, ev_[0], ev_[3])) != cudaSuccess) {
            timedValid = false;
            return cuda_fail(t, "kernel timing");
        }
    }
    return HPHC_OK;
}

int Executor::setup_device_loop(const std::vector<SetView>& sets, const int* setOf,
                                const double* params, int P) {
    if (P < 1) {
        error = "no problems to evaluate";
        return HPHC_ERR_BAD_ARGUMENT;
    }
    if (fixedR && fixedItems) {
        R = fixedR;
        itemsPerSM = fixedItems;
        tuned_ = true;
    }
    if (!tuned_) {
        const int st = autotune(sets, setOf, params, P, nullptr);
        if (st) return st;
    }
    wideBands_ = true;
    int st = build_plan(sets, setOf, params, P, nullptr, R, itemsPerSM);
    wideBands_ = false;
    if (st) return st;
    drop_graph();  // the tables' layout changed under any captured graph
    cudaError_t e;
    if ((e = cudaMemcpyAsync(dTables_, hStaging_, tablesBytes_, cudaMemcpyHostToDevice, stream_)))
        return cuda_fail(e, "stage tables");
    if (precision_ != HPHC_PRECISION_FP64) {
        char* d = static_cast<char*>(dTables_);
        if ((e = launch_pack_f32_jobs(D_, (int)plan_.pj.size(), plan_.maxN,
                                      reinterpret_cast<const PackJob*>(d + offPJ_), stream_)))
            return cuda_fail(e, "pack kernel");
    }
    if ((e = cudaStreamSynchronize(stream_))) return cuda_fail(e, "device loop set-up");
    loopGrid_ = sweep_grid(R);
    return HPHC_OK;
}

int Executor::enqueue_device_body() {
    const int prec = precision_ == HPHC_PRECISION_FP64 ? 0 : 1;
    char* d = static_cast<char*>(dTables_);
    const auto* sp = reinterpret_cast<const SweepProblem*>(d + offSP_);
    auto* items = reinterpret_cast<WorkItem*>(d + offItems_);
    const auto* nItems = reinterpret_cast<const int*>(d + offNItems_);
    const auto* fp = reinterpret_cast<const FinishProblem*>(d + offFP_);
    const auto* fb = reinterpret_cast<const FinishBlock*>(d + offFB_);
    cudaError_t e;
    if ((e = cudaMemsetAsync(dCounter_, 0, sizeof(int), stream_)))
        return cuda_fail(e, "reset work counter");
    // the plan lists every earlier tile for any sigma and omega: start each
    // item where the current constants allow a term
    if ((e = launch_band_starts((int)plan_.items.size(), sp, items, nItems, R, stream_)))
        return cuda_fail(e, "band kernel");
    if (colNeed_ && (e = cudaMemsetAsync(dColAcc_, 0, colNeed_ * sizeof(unsigned long long),
                                         stream_)))
        return cuda_fail(e, "reset column sums");
    if ((e = launch_sweep_list(prec, D_, R, variant_, loopGrid_, sp, items, nItems, dCounter_,
                               stream_)))
        return cuda_fail(e, "sweep kernel");
    if ((e = launch_finish_list(plan_.nBlocks, fp, fb, dBlockSums_, stream_)))
        return cuda_fail(e, "finish kernel");
    if ((e = launch_final_list(plan_.P, fp, dBlockSums_, dOut_, stream_)))
        return cuda_fail(e, "final kernel");
    lastLaunches = 4;
    return HPHC_OK;
}

SweepProblem* Executor::device_sweep_problems() const {
    return reinterpret_cast<SweepProblem*>(static_cast<char*>(dTables_) + offSP_);
}

FinishProblem* Executor::device_finish_problems() const {
    return reinterpret_cast<FinishProblem*>(static_cast<char*>(dTables_) + offFP_);
}

void Executor::count_terms(const std::vector<SetView>& sets, double* bTerms, double* sTerms,
                           double* bEvals) const {
    double nb = 0.0, ns = 0.0, ne = 0.0;
    const int stripEvents = kSweepThreads * R;
    for (const WorkItem& w : plan_.items) {
        const SetView& s = sets[plan_.setOf[w.problem]];
        const PairConsts& c = plan_.sp[w.problem].c;
        const int nTiles = plan_.sp[w.problem].nTiles;
        const int ts0 = w.strip * R, ts1 = std::min(ts0 + R, nTiles);
        double tminI = INFINITY, tmaxI = -INFINITY;
        for (int t = ts0; t < ts1; ++t) {
            tminI = std::min(tminI, s.hTileMin[t]);
            tmaxI = std::max(tmaxI, s.hTileMax[t]);
        }
        const double ni = std::min(stripEvents, s.N - w.strip * stripEvents);
        const bool sym = plan_.sp[w.problem].symmetric != 0;
        for (int jt = w.jt0; jt < w.jt1; ++jt) {
            bool b, se;
            tile_needs(tminI, tmaxI, s.hTileMin[jt], s.hTileMax[jt], c, &b, &se);
            if (sym && jt >= ts1) b = false;
            const double nj = std::min(kTile, s.N - jt * kTile);
            if (b) {
                // a symmetric tile also accounts for the pairs' other order
                nb += (sym && jt < ts0 ? 2.0 : 1.0) * ni * nj;
                ne += ni * nj;
            }
            if (se) ns += ni * nj;
        }
    }
    *bTerms = nb;
    *sTerms = ns;
    if (bEvals) *bEvals = ne;
}

}  // namespace hphc
