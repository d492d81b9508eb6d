// Tuning cache: launch shapes chosen by the autotuner, stored per key in a small versioned text file
// so later processes (and other handles on the same GPU model and index shape) start from them.
//
// Format:
//   tblaeq-tuning-cache 1
//   <key> TAB <levels> TAB <variant>:<grid percent>,<variant>:<grid percent>,...
// A file with another first line is not read (and is replaced on the next store). Stores rewrite
// the file through a temporary and a rename, so readers never see half a file.
#include "tuning.hpp"

#include <cstdio>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace tblaeq {

namespace {
const char* kHeader = "tblaeq-tuning-cache 1";

bool parseShapes(const std::string& text, size_t n, LaunchShapes& out) {
    out.variants.clear();
    out.gridPercent.clear();
    std::istringstream in(text);
    std::string item;
    while (std::getline(in, item, ',')) {
        const size_t c = item.find(':');
        if (c == std::string::npos) return false;
        try {
            out.variants.push_back(std::stoi(item.substr(0, c)));
            out.gridPercent.push_back(std::stoi(item.substr(c + 1)));
        } catch (const std::exception&) {
            return false;
        }
    }
    return out.variants.size() == n;
}

std::vector<std::pair<std::string, std::string>> readEntries(const std::string& path) {
    std::vector<std::pair<std::string, std::string>> entries;
    std::ifstream in(path);
    std::string line;
    if (!in || !std::getline(in, line) || line != kHeader) return entries;
    while (std::getline(in, line)) {
        const size_t t = line.find('\t');
        if (t == std::string::npos || t == 0) continue;
        entries.emplace_back(line.substr(0, t), line.substr(t + 1));
    }
    return entries;
}
}  // namespace

bool tuningLookup(const std::string& path, const std::string& key, LaunchShapes& out) {
    for (const auto& [k, rest] : readEntries(path)) {
        if (k != key) continue;
        const size_t t = rest.find('\t');
        if (t == std::string::npos) return false;
        size_t n = 0;
        try {
            n = std::stoul(rest.substr(0, t));
        } catch (const std::exception&) {
            return false;
        }
        return parseShapes(rest.substr(t + 1), n, out);
    }
    return false;
}

void tuningStore(const std::string& path, const std::string& key, const LaunchShapes& s) {
    if (key.empty() || key.find_first_of("\t\n\r") != std::string::npos)
        throw std::invalid_argument("tuning key must be non-empty without tabs or line breaks");
    if (s.variants.size() != s.gridPercent.size() || s.variants.empty())
        throw std::invalid_argument("tuning entry needs one variant and one grid percentage per level");
    std::ostringstream line;
    line << key << '\t' << s.variants.size() << '\t';
    for (size_t i = 0; i < s.variants.size(); ++i) line << (i ? "," : "") << s.variants[i] << ':' << s.gridPercent[i];
    auto entries = readEntries(path);
    bool replaced = false;
    for (auto& e : entries)
        if (e.first == key) {
            e.second = line.str().substr(key.size() + 1);
            replaced = true;
        }
    if (!replaced) entries.emplace_back(key, line.str().substr(key.size() + 1));
    const std::string tmp = path + ".tmp";
    {
        std::ofstream out(tmp, std::ios::trunc);
        if (!out) throw std::runtime_error("Cannot write: " + tmp);
        out << kHeader << '\n';
        for (const auto& [k, rest] : entries) out << k << '\t' << rest << '\n';
        if (!out) throw std::runtime_error("Short write: " + tmp);
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) throw std::runtime_error("Cannot write: " + path);
}

}  // namespace tblaeq
