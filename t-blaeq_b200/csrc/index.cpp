// Host index container: on-disk layout (byte-compatible with the reference's IndexSerializer)
// and the synthetic hierarchy generator (byte-compatible with the reference's --gen-index).
#include "index.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <filesystem>
#include <numeric>
#include <random>
#include <stdexcept>

namespace tblaeq {
namespace fs = std::filesystem;

namespace {

// ---------------------------------------------------------------------------------------------
// Raw little-endian file helpers. The reference writes fields back to back with no padding
// (src/core/IndexSerializer.cu:69-259), so every reader here checks the remaining length.
// ---------------------------------------------------------------------------------------------
struct Writer {
    FILE* f = nullptr;
    std::string path;
    explicit Writer(const std::string& p) : path(p) {
        f = std::fopen(p.c_str(), "wb");
        if (!f) throw std::runtime_error("Cannot write: " + p);
    }
    ~Writer() {
        if (f) std::fclose(f);
    }
    void bytes(const void* p, size_t n) {
        if (n && std::fwrite(p, 1, n, f) != n) throw std::runtime_error("Short write: " + path);
    }
    void u64(uint64_t v) { bytes(&v, 8); }
    void u8(uint8_t v) { bytes(&v, 1); }
};

struct Reader {
    FILE* f = nullptr;
    std::string path;
    uint64_t remaining = 0;
    explicit Reader(const std::string& p) : path(p) {
        f = std::fopen(p.c_str(), "rb");
        if (!f) throw std::runtime_error("Cannot read: " + p);
        std::error_code ec;
        remaining = fs::file_size(p, ec);
        if (ec) throw std::runtime_error("Cannot stat: " + p);
    }
    ~Reader() {
        if (f) std::fclose(f);
    }
    void bytes(void* p, uint64_t n) {
        if (n > remaining) throw std::runtime_error("Truncated index file: " + path);
        if (n && std::fread(p, 1, n, f) != n) throw std::runtime_error("Read error: " + path);
        remaining -= n;
    }
    uint64_t u64() {
        uint64_t v;
        bytes(&v, 8);
        return v;
    }
    uint8_t u8() {
        uint8_t v;
        bytes(&v, 1);
        return v;
    }
    // Element counts read from a header are checked against the bytes left before allocating.
    void expect(uint64_t count, uint64_t elemSize) {
        if (elemSize && count > remaining / elemSize) throw std::runtime_error("Truncated index file: " + path);
    }
};

// Lemire's fastmod for 32-bit operands: exact a % d for a, d < 2^32, d > 0.
struct FastMod32 {
    uint64_t M;
    uint32_t d;
    explicit FastMod32(uint32_t dd) : M(UINT64_C(0xFFFFFFFFFFFFFFFF) / dd + 1), d(dd) {}
    uint32_t operator()(uint32_t a) const {
        const uint64_t lowbits = M * a;
        return static_cast<uint32_t>((static_cast<__uint128_t>(lowbits) * d) >> 64);
    }
};

}  // namespace

void HostIndex::validate() const {
    auto fail = [](const std::string& m) { throw std::runtime_error("Invalid index: " + m); };
    if (D == 0) fail("D == 0");
    if (height < 2 || intervals != height - 1) fail("height/intervals mismatch");
    if (meshSizes.size() != height) fail("meshSizes length != height");
    if (ratios.size() != intervals) fail("ratios length != intervals");
    if (pTensors.size() != intervals || radius.size() != intervals) fail("per-interval arrays missing");
    if (maps.size() != height) fail("maps length != height");
    if (meshSizes[0] != N) fail("finest mesh size != N");
    for (uint64_t l = 0; l < intervals; ++l) {
        const PTensor& P = pTensors[l];
        if (P.D != D) fail("P-tensor D mismatch at interval " + std::to_string(l));
        if (P.cols != meshCount(l) || P.rows != meshCount(l + 1) || P.nnz != P.rows)
            fail("P-tensor shape mismatch at interval " + std::to_string(l));
        if (P.colRes.size() != P.cols + 1 || P.nnzPerCol.size() != P.cols || P.rowIds.size() != P.nnz ||
            P.vals.size() != P.nnz * D)
            fail("P-tensor array sizes at interval " + std::to_string(l));
        if (P.colRes[0] != 0 || P.colRes[P.cols] != P.nnz) fail("colRes endpoints at interval " + std::to_string(l));
        for (uint64_t c = 0; c < P.cols; ++c) {
            if (P.colRes[c + 1] < P.colRes[c] || P.colRes[c + 1] - P.colRes[c] != P.nnzPerCol[c])
                fail("colRes/nnzPerCol mismatch at interval " + std::to_string(l));
        }
        for (uint64_t j = 0; j < P.nnz; ++j) {
            if (P.rowIds[j] != j) fail("non-identity rowIds at interval " + std::to_string(l));
        }
        if (radius[l].size() != P.cols) fail("radius length at interval " + std::to_string(l));
    }
    for (uint64_t m = 1; m < height; ++m) {
        if (maps[m].size() != meshCount(m)) fail("map length at mesh " + std::to_string(m));
        for (uint64_t v : maps[m]) {
            if (v >= meshCount(m)) fail("map entry out of range at mesh " + std::to_string(m));
        }
    }
    if (coarsest.dim != D || coarsest.nnz != meshCount(0) || coarsest.ids.size() != coarsest.nnz ||
        coarsest.vals.size() != coarsest.nnz * D)
        fail("coarsest mesh shape");
    for (uint64_t i = 0; i < coarsest.nnz; ++i) {
        if (coarsest.ids[i] >= meshCount(0)) fail("coarsest id out of range");
    }
}

// ---------------------------------------------------------------------------------------------
// Serializer (layout of src/core/IndexSerializer.cu:69-235)
// ---------------------------------------------------------------------------------------------
void saveIndex(const HostIndex& d, const std::string& dir) {
    fs::create_directories(dir);
    {
        Writer w(dir + "/metadata.bin");
        w.u64(d.D);
        w.u64(d.N);
        w.u64(d.height);
        w.u64(d.intervals);
        w.u8(d.isAos);
        for (uint64_t i = 0; i < d.intervals; ++i) w.u64(d.ratios[i]);
        w.u64(d.meshSizes.size());
        w.bytes(d.meshSizes.data(), d.meshSizes.size() * 8);
    }
    for (uint64_t i = 0; i < d.intervals; ++i) {
        const PTensor& t = d.pTensors[i];
        Writer w(dir + "/P_Tensor_" + std::to_string(i) + ".bin");
        w.u64(t.D);
        w.u64(t.rows);
        w.u64(t.cols);
        w.u64(t.nnz);
        w.u8(t.isAos);
        w.bytes(t.rowIds.data(), t.nnz * 8);
        w.bytes(t.nnzPerCol.data(), t.cols * 8);
        w.bytes(t.colRes.data(), (t.cols + 1) * 8);
        w.bytes(t.vals.data(), t.nnz * t.D * 8);
    }
    for (uint64_t i = 0; i < d.intervals; ++i) {
        Writer w(dir + "/MaxRadius_" + std::to_string(i) + ".bin");
        const uint64_t count = d.meshSizes[d.intervals - i];
        w.u64(count);
        w.bytes(d.radius[i].data(), count * 8);
    }
    for (uint64_t m = 1; m < d.height; ++m) {
        if (d.maps[m].empty()) continue;
        Writer w(dir + "/Map_" + std::to_string(m) + ".bin");
        w.u64(d.maps[m].size());
        w.bytes(d.maps[m].data(), d.maps[m].size() * 8);
    }
    {
        Writer w(dir + "/Coreast_Mesh.bin");
        w.u64(d.coarsest.rows);
        w.u64(d.coarsest.dim);
        w.u64(d.coarsest.nnz);
        w.u8(d.coarsest.isAos);
        w.bytes(d.coarsest.ids.data(), d.coarsest.nnz * 8);
        w.bytes(d.coarsest.vals.data(), d.coarsest.nnz * d.coarsest.dim * 8);
    }
}

HostIndex loadIndex(const std::string& dir) {
    HostIndex d;
    {
        Reader r(dir + "/metadata.bin");
        d.D = r.u64();
        d.N = r.u64();
        d.height = r.u64();
        d.intervals = r.u64();
        d.isAos = r.u8();
        if (d.height < 2 || d.height > 64 || d.intervals != d.height - 1)
            throw std::runtime_error("Invalid index: bad height in " + dir + "/metadata.bin");
        d.ratios.resize(d.intervals);
        for (auto& v : d.ratios) v = r.u64();
        const uint64_t msz = r.u64();
        if (msz != d.height) throw std::runtime_error("Invalid index: meshSizes length in metadata.bin");
        d.meshSizes.resize(msz);
        r.bytes(d.meshSizes.data(), msz * 8);
    }
    d.pTensors.resize(d.intervals);
    d.radius.resize(d.intervals);
    d.maps.resize(d.height);
    for (uint64_t i = 0; i < d.intervals; ++i) {
        PTensor& t = d.pTensors[i];
        Reader r(dir + "/P_Tensor_" + std::to_string(i) + ".bin");
        t.D = r.u64();
        t.rows = r.u64();
        t.cols = r.u64();
        t.nnz = r.u64();
        t.isAos = r.u8();
        if (t.D != d.D) throw std::runtime_error("Invalid index: P-tensor D mismatch in " + r.path);
        r.expect(t.nnz, 8);
        t.rowIds.resize(t.nnz);
        r.bytes(t.rowIds.data(), t.nnz * 8);
        r.expect(t.cols, 8);
        t.nnzPerCol.resize(t.cols);
        r.bytes(t.nnzPerCol.data(), t.cols * 8);
        t.colRes.resize(t.cols + 1);
        r.bytes(t.colRes.data(), (t.cols + 1) * 8);
        r.expect(t.nnz, 8 * t.D);
        t.vals.resize(t.nnz * t.D);
        r.bytes(t.vals.data(), t.nnz * t.D * 8);
    }
    for (uint64_t i = 0; i < d.intervals; ++i) {
        Reader r(dir + "/MaxRadius_" + std::to_string(i) + ".bin");
        const uint64_t count = r.u64();
        r.expect(count, 8);
        d.radius[i].resize(count);
        r.bytes(d.radius[i].data(), count * 8);
    }
    for (uint64_t m = 1; m < d.height; ++m) {
        const std::string path = dir + "/Map_" + std::to_string(m) + ".bin";
        if (!fs::exists(path)) continue;
        Reader r(path);
        const uint64_t n = r.u64();
        r.expect(n, 8);
        d.maps[m].resize(n);
        r.bytes(d.maps[m].data(), n * 8);
    }
    {
        Reader r(dir + "/Coreast_Mesh.bin");
        d.coarsest.rows = r.u64();
        d.coarsest.dim = r.u64();
        d.coarsest.nnz = r.u64();
        d.coarsest.isAos = r.u8();
        r.expect(d.coarsest.nnz, 8);
        d.coarsest.ids.resize(d.coarsest.nnz);
        r.bytes(d.coarsest.ids.data(), d.coarsest.nnz * 8);
        r.expect(d.coarsest.nnz, 8 * d.coarsest.dim);
        d.coarsest.vals.resize(d.coarsest.nnz * d.coarsest.dim);
        r.bytes(d.coarsest.vals.data(), d.coarsest.nnz * d.coarsest.dim * 8);
    }
    d.datasetName = fs::path(dir).filename().string();
    if (d.datasetName.empty()) d.datasetName = fs::path(dir).parent_path().filename().string();
    d.validate();
    return d;
}

// ---------------------------------------------------------------------------------------------
// Synthetic hierarchy generator
// ---------------------------------------------------------------------------------------------
HostIndex generateRandomIndex(const GenParams& p) {
    if (p.height < 2) throw std::invalid_argument("QueryHandler: height must be >= 2");
    if (p.ratios.size() != p.height - 1) throw std::invalid_argument("QueryHandler: ratios size must equal height - 1");
    if (p.D == 0 || p.N == 0) throw std::invalid_argument("generateRandomIndex: N and D must be > 0");
    if (p.valMin <= 0.0) throw std::invalid_argument("RandomKmeans: valMin must be > 0");
    if (p.valMin >= p.valMax) throw std::invalid_argument("RandomKmeans: valMin must be < valMax");
    if (p.sigmaDivisor <= 0.0) throw std::invalid_argument("RandomKmeans: sigmaDivisor must be > 0");
    for (uint64_t r : p.ratios) {
        if (r == 0) throw std::invalid_argument("Invalid --ratios: ratio must be > 0");
    }
    if (p.N >= (UINT64_C(1) << 32)) throw std::invalid_argument("generateRandomIndex: N must be < 2^32");

    // Build-plan truncation: stop at the first interval whose coarse mesh would hold one node.
    std::vector<uint64_t> ratios;
    {
        uint64_t n = p.N;
        size_t keep = p.ratios.size();
        for (size_t i = 0; i < p.ratios.size(); ++i) {
            const uint64_t c = (n / p.ratios[i] == 0) ? 1 : n / p.ratios[i];
            if (c == 1) {
                keep = i + 1;
                break;
            }
            n = c;
        }
        ratios.assign(p.ratios.begin(), p.ratios.begin() + static_cast<long>(keep));
    }
    const uint64_t intervals = ratios.size();
    const uint64_t height = intervals + 1;
    const uint64_t D = p.D;

    // Layer sizes, finest (0) .. coarsest (intervals).
    std::vector<uint64_t> sizes(intervals + 1);
    sizes[0] = p.N;
    for (uint64_t i = 0; i < intervals; ++i) sizes[i + 1] = std::max<uint64_t>(1, sizes[i] / ratios[i]);

    auto roundIfNeeded = [&](double v) { return p.isInt ? std::round(v) : v; };

    // layers[i] = flat AOS coordinates of layer i (finest = 0).
    std::vector<std::vector<double>> layers(intervals + 1);
    std::mt19937_64 rng(p.seed);
    {
        std::uniform_real_distribution<double> uni(p.valMin, p.valMax);
        auto& top = layers[intervals];
        top.resize(sizes[intervals] * D);
        for (uint64_t i = 0; i < sizes[intervals]; ++i)
            for (uint64_t d = 0; d < D; ++d) top[i * D + d] = roundIfNeeded(uni(rng));
    }
    for (uint64_t lvl = intervals; lvl > 0; --lvl) {
        const auto& parents = layers[lvl];
        const uint64_t nP = sizes[lvl];
        const uint64_t nC = sizes[lvl - 1];
        const double spacing =
            (p.valMax - p.valMin) / std::pow(static_cast<double>(nP), 1.0 / static_cast<double>(D));
        const double sigma = spacing / p.sigmaDivisor;
        std::normal_distribution<double> normal(0.0, sigma);
        auto& children = layers[lvl - 1];
        children.resize(nC * D);
        for (uint64_t ci = 0; ci < nC; ++ci) {
            const double* par = &parents[(ci % nP) * D];
            double* ch = &children[ci * D];
            for (uint64_t d = 0; d < D; ++d) {
                double v = par[d] + normal(rng);
                v = std::clamp(v, p.valMin, p.valMax);
                ch[d] = roundIfNeeded(v);
            }
        }
    }

    HostIndex idx;
    idx.D = D;
    idx.N = p.N;
    idx.height = height;
    idx.intervals = intervals;
    idx.isAos = 1;
    idx.ratios = ratios;
    idx.pTensors.resize(intervals);
    idx.radius.resize(intervals);
    idx.maps.resize(height);

    // Fine -> coarse: layer i (fine, mesh index intervals - i) clustered into layer i + 1.
    for (uint64_t i = 0; i < intervals; ++i) {
        const uint64_t nF = sizes[i];
        const uint64_t nP = sizes[i + 1];
        const uint64_t fineMesh = intervals - i;
        const uint64_t pIdx = fineMesh - 1;
        idx.meshSizes.push_back(nF);
        const std::vector<double>& fine = layers[i];
        const std::vector<double>& coarse = layers[i + 1];

        PTensor& P = idx.pTensors[pIdx];
        P.D = D;
        P.rows = nF;
        P.cols = nP;
        P.nnz = nF;
        P.isAos = 1;
        P.nnzPerCol.assign(nP, 0);
        for (uint64_t ci = 0; ci < nF; ++ci) ++P.nnzPerCol[ci % nP];
        P.colRes.assign(nP + 1, 0);
        for (uint64_t c = 1; c <= nP; ++c) P.colRes[c] = P.colRes[c - 1] + P.nnzPerCol[c - 1];
        P.rowIds.resize(nF);
        std::iota(P.rowIds.begin(), P.rowIds.end(), uint64_t{0});

        // Sort-to-original map: the index permutation std::sort produces when ordering the
        // fine nodes by their parent label (labels[ci] = ci % nP).
        std::vector<uint64_t> order(nF);
        std::iota(order.begin(), order.end(), uint64_t{0});
        const FastMod32 mod(static_cast<uint32_t>(nP));
        std::sort(order.begin(), order.end(), [&mod](uint64_t a, uint64_t b) {
            return mod(static_cast<uint32_t>(a)) < mod(static_cast<uint32_t>(b));
        });

        P.vals.resize(nF * D);
        idx.radius[pIdx].resize(nP);
        for (uint64_t c = 0; c < nP; ++c) {
            const double* cv = &coarse[c * D];
            double maxDist = 0.0;
            for (uint64_t pos = P.colRes[c]; pos < P.colRes[c + 1]; ++pos) {
                const double* fv = &fine[order[pos] * D];
                double* out = &P.vals[pos * D];
                double sum = 0.0;
                for (uint64_t d = 0; d < D; ++d) {
                    out[d] = fv[d] / cv[d];
                    const double diff = cv[d] - fv[d];
                    sum += diff * diff;
                }
                maxDist = std::max(maxDist, std::sqrt(sum));
            }
            idx.radius[pIdx][c] = maxDist;
        }
        idx.maps[fineMesh] = std::move(order);

        if (i + 2 == height) {
            idx.meshSizes.push_back(nP);
            idx.coarsest.rows = nP;
            idx.coarsest.dim = D;
            idx.coarsest.nnz = nP;
            idx.coarsest.isAos = 1;
            idx.coarsest.ids.resize(nP);
            std::iota(idx.coarsest.ids.begin(), idx.coarsest.ids.end(), uint64_t{0});
            idx.coarsest.vals = coarse;
        }
        // The fine layer is no longer needed once its P-tensor and radii exist.
        std::vector<double>().swap(layers[i]);
    }
    idx.datasetName = "Gen" + std::to_string(p.N) + "D" + std::to_string(D);
    return idx;
}

void loadPointsText(const std::string& path, uint64_t& n, uint64_t& d, std::vector<double>* points) {
    std::unique_ptr<FILE, int (*)(FILE*)> f(std::fopen(path.c_str(), "r"), &std::fclose);
    if (!f) throw std::runtime_error("loadFromFile: cannot open '" + path + "'");
    struct LineBuf {
        char* p = nullptr;
        size_t cap = 0;
        ~LineBuf() { std::free(p); }
    } buf;
    char*& line = buf.p;
    auto next = [&]() -> bool { return getline(&buf.p, &buf.cap, f.get()) >= 0; };
    if (!next()) throw std::runtime_error("loadFromFile: empty file '" + path + "'");
    {
        // Two integers, both positive (the reference reads them as int).
        char* end = nullptr;
        const long long a = std::strtoll(line, &end, 10);
        char* end2 = nullptr;
        const long long b = (end != line) ? std::strtoll(end, &end2, 10) : 0;
        if (end == line || end2 == end || a <= 0 || b <= 0 || a > 0x7fffffffLL || b > 0x7fffffffLL)
            throw std::runtime_error("loadFromFile: invalid header in '" + path + "'");
        n = static_cast<uint64_t>(a);
        d = static_cast<uint64_t>(b);
    }
    if (!points) return;
    points->assign(n * d, 0.0);
    uint64_t row = 0;
    while (row < n && next()) {
        char* p = line;
        uint64_t col = 0;
        while (col < d) {
            char* end = nullptr;
            const double v = std::strtod(p, &end);
            if (end == p) break;
            (*points)[row * d + col++] = v;
            p = end;
        }
        if (col != d) throw std::runtime_error("loadFromFile: dimension mismatch at row " + std::to_string(row + 1));
        ++row;
    }
    if (row != n) throw std::runtime_error("loadFromFile: row count mismatch in '" + path + "'");
}

}  // namespace tblaeq
