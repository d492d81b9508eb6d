// Tuning cache of autotuned launch shapes (see tuning.cpp for the file format).
#pragma once

#include <string>
#include <vector>

namespace tblaeq {

// Launch shape per expand launch (one per mesh of the index): kernel variant and persistent grid
// as a percentage of full occupancy.
struct LaunchShapes {
    std::vector<int> variants;
    std::vector<int> gridPercent;
};

// Looks `key` up in the cache file at `path`; false when the file, the key or a valid entry is missing.
bool tuningLookup(const std::string& path, const std::string& key, LaunchShapes& out);
// Adds or replaces the entry for `key` (creates the file when needed).
void tuningStore(const std::string& path, const std::string& key, const LaunchShapes& shapes);

}  // namespace tblaeq
