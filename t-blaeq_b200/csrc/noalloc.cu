// Allocation-free variant of the per-level range step (tblaeq_level_range_noalloc).
//
// Some callers cannot allocate device memory while they query: a caller that runs inside a
// pre-sized memory pool (a serving process that reserved its whole budget at start-up), a caller
// whose allocations are forbidden between start-up and shutdown by its own rules, or code running
// where cudaMalloc would synchronise the device at a bad moment. tblaeq_level allocates its level
// buffers on first use; this variant allocates nothing: the caller passes the input grid and the
// output buffers, and every piece of scratch lives in one file-scope __device__ array of fixed size.
//
// Limits: at most kNoAllocMaxGrid input entries, at most kNoAllocMaxOut output entries and D <= 16
// (the scratch below is sized for exactly that). Every GPU that loads this library holds the array
// until the process exits.
//
// Sharing: all calls on a device use the same array, and it keeps the previous call's contents.
// The control words that must start at zero are cleared at the start of every call. Calls whose
// work overlaps on the GPU (different streams or handles on the same device) race on the array;
// callers must serialise them.
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "../../include/tblaeq.h"
#include "handler.hpp"
#include "noalloc.hpp"

namespace tblaeq {

namespace {

constexpr uint64_t kMaxD = 16;
constexpr uint64_t kTilesIn = (kNoAllocMaxGrid + kWarpTile - 1) / kWarpTile + 2;
constexpr uint64_t kTilesOut = (kNoAllocMaxOut + kWarpTile - 1) / kWarpTile + 2;

// Byte layout of the scratch array (all offsets 256-byte aligned).
constexpr uint64_t align256(uint64_t v) { return (v + 255) & ~uint64_t(255); }
constexpr uint64_t kOffCtrl = 0;                                             // zeroed every call
constexpr uint64_t kCtrlDesc = 0;                                            // 2 launches of descriptors
constexpr uint64_t kCtrlTickets = kCtrlDesc + 2 * kTilesOut * 8;             // 2 tickets
constexpr uint64_t kCtrlStatus = kCtrlTickets + 16;
constexpr uint64_t kCtrlHdr = kCtrlStatus + 16;                              // 3 headers x 2 words
constexpr uint64_t kCtrlBytes = align256(kCtrlHdr + 32);
constexpr uint64_t kOffBox = kOffCtrl + kCtrlBytes;                          // lo|hi of the query
constexpr uint64_t kOffRoot = align256(kOffBox + 2 * kMaxD * 8);             // root frontier (1 entry)
constexpr uint64_t kRootBytes = align256(4 * 4 + kMaxD * 8 + 16) + align256(kTilesIn * 4);
constexpr uint64_t kOffSurv = kOffRoot + kRootBytes;                         // survivors of the level
constexpr uint64_t kSurvQ = 0;
constexpr uint64_t kSurvNode = align256(kNoAllocMaxGrid * 4);
constexpr uint64_t kSurvCbeg = kSurvNode + align256(kNoAllocMaxGrid * 4);
constexpr uint64_t kSurvCpre = kSurvCbeg + align256(kNoAllocMaxGrid * 4);
constexpr uint64_t kSurvX = kSurvCpre + align256(kNoAllocMaxGrid * 4);
constexpr uint64_t kSurvTiles = kSurvX + align256(kNoAllocMaxGrid * kMaxD * 8);
constexpr uint64_t kSurvBytes = kSurvTiles + align256(kTilesOut * 4);
constexpr uint64_t kScratchBytes = kOffSurv + kSurvBytes;

// The scratch itself: one copy per device that loads the library.
__device__ __align__(256) unsigned char gNoAllocScratch[kScratchBytes];

// Device address of gNoAllocScratch per device ordinal, looked up once per device.
std::mutex gScratchMutex;
unsigned char* gScratchAddr[64] = {};

unsigned char* scratchForCurrentDevice() {
    int dev = 0;
    TBLAEQ_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw std::invalid_argument("device ordinal out of range");
    std::lock_guard<std::mutex> g(gScratchMutex);
    if (!gScratchAddr[dev]) {
        void* p = nullptr;
        TBLAEQ_CUDA(cudaGetSymbolAddress(&p, gNoAllocScratch));
        gScratchAddr[dev] = static_cast<unsigned char*>(p);
    }
    return gScratchAddr[dev];
}

}  // namespace

uint64_t noAllocScratchBytes() { return kScratchBytes; }

uint64_t runLevelRangeNoAlloc(Runtime& rt, uint64_t l, const uint64_t* dIds, const double* dVals, uint64_t p,
                              const double* lo, const double* hi, uint64_t* outIds, double* outVals,
                              uint64_t outCap) {
    const DeviceIndex& di = *rt.dev;
    const uint64_t D = di.D;
    if (l >= di.intervals) throw std::out_of_range("level out of range");
    if (D > kMaxD) throw std::invalid_argument("no-alloc level step supports D <= 16");
    if (p > kNoAllocMaxGrid)
        throw std::invalid_argument("no-alloc level step: grid larger than " + std::to_string(kNoAllocMaxGrid));
    if (outCap > kNoAllocMaxOut)
        throw std::invalid_argument("no-alloc level step: output capacity above " + std::to_string(kNoAllocMaxOut));
    if (p == 0) return 0;
    unsigned char* s = scratchForCurrentDevice();
    cudaStream_t st = rt.stream;

    auto* desc = reinterpret_cast<unsigned long long*>(s + kOffCtrl + kCtrlDesc);
    auto* tickets = reinterpret_cast<uint32_t*>(s + kOffCtrl + kCtrlTickets);
    auto* status = reinterpret_cast<uint32_t*>(s + kOffCtrl + kCtrlStatus);
    auto* hdr = reinterpret_cast<uint32_t*>(s + kOffCtrl + kCtrlHdr);
    auto* box = reinterpret_cast<double*>(s + kOffBox);
    unsigned char* root = s + kOffRoot;
    auto* rq = reinterpret_cast<uint32_t*>(root);
    auto* rcbeg = rq + 1;
    auto* rcpre = rq + 2;
    auto* rx = reinterpret_cast<double*>(root + 16);
    auto* rtiles = reinterpret_cast<uint32_t*>(root + align256(4 * 4 + kMaxD * 8 + 16));
    unsigned char* sv = s + kOffSurv;

    TBLAEQ_CUDA(cudaMemsetAsync(s + kOffCtrl, 0, kCtrlBytes, st));
    TBLAEQ_CUDA(cudaMemcpyAsync(box, lo, D * 8, cudaMemcpyHostToDevice, st));
    TBLAEQ_CUDA(cudaMemcpyAsync(box + D, hi, D * 8, cudaMemcpyHostToDevice, st));
    launchRootFrontier(rq, rcbeg, rcpre, rx, rtiles, hdr, 1, static_cast<uint32_t>(p), static_cast<int>(D), kWarpTile,
                       st);

    ExpandArgs a{};
    a.in = FrontierIn{rq, rcbeg, rcpre, rx, rtiles, hdr, 1u, static_cast<uint32_t>(kTilesIn)};
    a.child.rows = dVals;
    a.child.keys = dIds;
    a.child.nodes = di.nodeOrig[l].as<NodeRec>();
    a.query.boxes = box;
    a.fout = FrontierOut{reinterpret_cast<uint32_t*>(sv + kSurvQ),    reinterpret_cast<uint32_t*>(sv + kSurvNode),
                         reinterpret_cast<uint32_t*>(sv + kSurvCbeg), reinterpret_cast<uint32_t*>(sv + kSurvCpre),
                         reinterpret_cast<double*>(sv + kSurvX),      reinterpret_cast<uint32_t*>(sv + kSurvTiles),
                         hdr + 2,                                     static_cast<uint32_t>(kNoAllocMaxGrid),
                         static_cast<uint32_t>(kTilesOut)};
    a.scratch.desc = desc;
    a.scratch.ticket = tickets;
    a.scratch.status = status;
    a.D = static_cast<int>(D);
    a.useFma = 1;
    launchExpand(a, kPredRangeRadius, false, 0, st);

    ExpandArgs b{};
    b.in = FrontierIn{reinterpret_cast<uint32_t*>(sv + kSurvQ),    reinterpret_cast<uint32_t*>(sv + kSurvCbeg),
                      reinterpret_cast<uint32_t*>(sv + kSurvCpre), reinterpret_cast<double*>(sv + kSurvX),
                      reinterpret_cast<uint32_t*>(sv + kSurvTiles), hdr + 2,
                      static_cast<uint32_t>(kNoAllocMaxGrid),      static_cast<uint32_t>(kTilesOut)};
    b.child.rows = di.rows[l];
    b.child.rowsOnHost = di.rowsOnHost[l];
    b.child.outMap = di.mapPtr[l + 1];
    b.rout.ids = outIds;
    b.rout.vals = outVals;
    b.rout.hdr = hdr + 4;
    b.rout.cap = static_cast<uint32_t>(outCap);
    b.scratch.desc = desc + kTilesOut;
    b.scratch.ticket = tickets + 1;
    b.scratch.status = status;
    b.D = static_cast<int>(D);
    b.useFma = 1;
    launchExpand(b, kPredAll, true, 0, st);

    uint32_t h[6] = {0, 0, 0, 0, 0, 0};
    uint32_t stWord = 0;
    TBLAEQ_CUDA(cudaMemcpyAsync(h, hdr, sizeof(h), cudaMemcpyDeviceToHost, st));
    TBLAEQ_CUDA(cudaMemcpyAsync(&stWord, status, 4, cudaMemcpyDeviceToHost, st));
    TBLAEQ_CUDA(cudaStreamSynchronize(st));
    if (stWord & (kStatusLookbackTimeout | kStatusWindowOverflow))
        throw CudaError(cudaErrorLaunchTimeout, "traversal kernel reported status " + std::to_string(stWord));
    // h[3]: children the survivors generate (what the caller's buffers must hold); h[4]: results
    // written. When the first launch overflowed, the second returned early and h[4] is 0.
    if (h[3] > kNoAllocMaxOut) throw NoAllocOverflow(h[3]);
    if (stWord) throw NoAllocOverflow(std::max(h[3], h[4]));
    return h[4];
}

}  // namespace tblaeq
