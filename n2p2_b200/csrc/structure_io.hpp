// input.data reader for whole files (Structure::readFromLines,
// reference src/libnnp/Structure.cpp:142-271, applied block by block as
// Dataset / Prediction read their structure files): all structures into flat
// arrays ready for Batch::setStructures.  Numbers are converted with correct
// rounding (std::from_chars; strtod for out-of-range values), so they are
// bit-identical to what the reference's atof reads.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace n2p2b200 {

struct StructureSet
{
    std::vector<int64_t> atomBegin{0};    // [S+1]
    std::vector<double> positions;        // [N][3]
    std::vector<double> forces;           // [N][3] reference forces
    std::vector<double> atomCharges;      // [N]
    std::vector<std::string> elements;    // [N] symbols
    std::vector<double> boxes;            // [S][3][3] (zeros when not periodic)
    std::vector<int32_t> periodic;        // [S]
    std::vector<double> energies;         // [S] reference energies
    std::vector<double> charges;          // [S] reference total charges
    std::vector<std::string> comments;    // [S]
    int64_t numStructures() const { return (int64_t)periodic.size(); }
    int64_t numAtoms() const { return atomBegin.back(); }
};

// Reads up to `limit` structures (all when limit < 0) from `text`
// (`length` bytes); throws std::runtime_error with the reference's messages.
void readStructures(const char* text, size_t length, int64_t limit, StructureSet& out);
void readStructuresFile(std::string const& fileName, int64_t limit, StructureSet& out);

} // namespace n2p2b200
