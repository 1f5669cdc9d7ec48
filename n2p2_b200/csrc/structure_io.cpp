// input.data reader (see structure_io.hpp).
#include "structure_io.hpp"

#include <algorithm>
#include <charconv>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <stdexcept>
#include <system_error>
#include <thread>

namespace n2p2b200 {

namespace {

struct Token
{
    const char* p;
    size_t n;
    bool is(char const* w) const { return std::strlen(w) == n && std::memcmp(p, w, n) == 0; }
    std::string str() const { return std::string(p, n); }
};

inline bool space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\f' || c == '\v'; }

// Tokens of the line [b, e).
void split(const char* b, const char* e, std::vector<Token>& out)
{
    out.clear();
    const char* p = b;
    while (p < e)
    {
        while (p < e && space(*p)) ++p;
        if (p >= e) break;
        const char* q = p;
        while (q < e && !space(*q)) ++q;
        out.push_back({p, (size_t)(q - p)});
        p = q;
    }
}

// Correctly rounded decimal -> double over exactly the token (std::from_chars,
// the same value strtod gives; a leading '+' is accepted as strtod does).
// Like atof, a token that is not a number reads as 0.
inline double number(std::vector<Token> const& w, size_t k)
{
    if (k >= w.size()) throw std::out_of_range("ERROR: Missing value in structure line.\n");
    const char* p = w[k].p;
    const char* e = p + w[k].n;
    if (p < e && *p == '+') ++p;
    double v = 0.0;
    auto r = std::from_chars(p, e, v);
    if (r.ec == std::errc::result_out_of_range) return std::strtod(w[k].p, nullptr);   // strtod's inf / denormal
    return r.ec == std::errc() ? v : 0.0;
}

struct Block
{
    std::vector<double> box, pos, force, q;
    std::vector<std::string> el;
    std::string comment;
    double energy = 0.0, charge = 0.0;
    void clear()
    {
        box.clear();
        pos.clear();
        force.clear();
        q.clear();
        el.clear();
        comment.clear();
        energy = charge = 0.0;
    }
};

void commit(Block const& b, StructureSet& out)
{
    const int64_t n = (int64_t)b.el.size();
    out.atomBegin.push_back(out.atomBegin.back() + n);
    out.positions.insert(out.positions.end(), b.pos.begin(), b.pos.end());
    out.forces.insert(out.forces.end(), b.force.begin(), b.force.end());
    out.atomCharges.insert(out.atomCharges.end(), b.q.begin(), b.q.end());
    out.elements.insert(out.elements.end(), b.el.begin(), b.el.end());
    const bool periodic = b.box.size() == 9;
    for (int k = 0; k < 9; ++k) out.boxes.push_back(periodic ? b.box[k] : 0.0);
    out.periodic.push_back(periodic ? 1 : 0);
    out.energies.push_back(b.energy);
    out.charges.push_back(b.charge);
    out.comments.push_back(b.comment);
}

} // namespace

namespace {

bool readRange(const char* text, size_t length, int64_t limit, StructureSet& out);

// Start of the first line at or after `p` whose first token is "begin".
const char* nextBegin(const char* p, const char* end)
{
    while (p < end)
    {
        const char* q = p;
        while (q < end && space(*q)) ++q;
        if (end - q >= 5 && std::memcmp(q, "begin", 5) == 0 && (end - q == 5 || space(q[5]) || q[5] == '\n'))
            return p;
        const char* eol = (const char*)std::memchr(p, '\n', (size_t)(end - p));
        if (!eol) return end;
        p = eol + 1;
    }
    return end;
}

void append(StructureSet& a, StructureSet const& b)
{
    const int64_t base = a.atomBegin.back();
    for (size_t k = 1; k < b.atomBegin.size(); ++k) a.atomBegin.push_back(base + b.atomBegin[k]);
    a.positions.insert(a.positions.end(), b.positions.begin(), b.positions.end());
    a.forces.insert(a.forces.end(), b.forces.begin(), b.forces.end());
    a.atomCharges.insert(a.atomCharges.end(), b.atomCharges.begin(), b.atomCharges.end());
    a.elements.insert(a.elements.end(), b.elements.begin(), b.elements.end());
    a.boxes.insert(a.boxes.end(), b.boxes.begin(), b.boxes.end());
    a.periodic.insert(a.periodic.end(), b.periodic.begin(), b.periodic.end());
    a.energies.insert(a.energies.end(), b.energies.begin(), b.energies.end());
    a.charges.insert(a.charges.end(), b.charges.begin(), b.charges.end());
    a.comments.insert(a.comments.end(), b.comments.begin(), b.comments.end());
}

} // namespace

// Large files without a limit are cut at "begin" lines into one range per
// host thread; the ranges are read concurrently and joined in file order
// (the first error in file order is the one reported).
void readStructures(const char* text, size_t length, int64_t limit, StructureSet& out)
{
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (limit >= 0 || length < (8u << 20) || hw == 1)
    {
        readRange(text, length, limit, out);
        return;
    }
    const char* end = text + length;
    std::vector<const char*> cut{text};
    for (unsigned t = 1; t < hw; ++t)
    {
        const char* c = nextBegin(std::max(cut.back(), text + length / hw * t), end);
        if (c > cut.back() && c < end) cut.push_back(c);
    }
    cut.push_back(end);
    const size_t R = cut.size() - 1;
    std::vector<StructureSet> part(R);
    std::vector<std::string> err(R);
    std::vector<int> errKind(R, 0);
    std::vector<char> open(R, 0);
    std::vector<std::thread> pool;
    for (size_t r = 0; r < R; ++r)
        pool.emplace_back([&, r] {
            try
            {
                open[r] = readRange(cut[r], (size_t)(cut[r + 1] - cut[r]), -1, part[r]) ? 1 : 0;
            }
            catch (std::out_of_range const& e)
            {
                err[r] = e.what();
                errKind[r] = 2;
            }
            catch (std::exception const& e)
            {
                err[r] = e.what();
                errKind[r] = 1;
            }
        });
    for (auto& th : pool) th.join();
    // a block left open before a cut ("begin" inside a block) continues past
    // it in a sequential read: read the file sequentially then
    for (size_t r = 0; r + 1 < R; ++r)
        if (open[r] && !errKind[r])
        {
            readRange(text, length, -1, out);
            return;
        }
    for (size_t r = 0; r < R; ++r)
    {
        if (errKind[r] == 2) throw std::out_of_range(err[r]);
        if (errKind[r] == 1) throw std::runtime_error(err[r]);
    }
    out = StructureSet{};
    for (size_t r = 0; r < R; ++r) append(out, part[r]);
}

namespace {

// Reads the blocks of [text, text + length); returns whether the range ended
// inside a block (a trailing block without "end", which is not read).
bool readRange(const char* text, size_t length, int64_t limit, StructureSet& out)
{
    out = StructureSet{};
    std::vector<Token> w;
    Block blk;
    bool inBlock = false;
    const char* p = text;
    const char* end = text + length;
    while (p < end && (limit < 0 || out.numStructures() < limit))
    {
        const char* eol = (const char*)std::memchr(p, '\n', (size_t)(end - p));
        if (!eol) eol = end;
        const char* lineBegin = p;
        split(p, eol, w);
        p = eol + 1;
        if (w.empty()) continue;   // blank lines are skipped
        Token const& k = w[0];
        if (!inBlock)
        {
            if (!k.is("begin")) throw std::runtime_error("ERROR: Unexpected line content, expected \"begin\" keyword.\n");
            inBlock = true;
            blk.clear();
        }
        if (k.is("begin"))
        {
            for (size_t i = 1; i < w.size(); ++i)
                if (!w[i].is("set=train") && !w[i].is("set=test"))
                    throw std::runtime_error("ERROR: Unknown keyword in structure specification, check \"begin\" "
                                             "arguments.\n");
        }
        else if (k.is("comment"))
        {
            // the line without the keyword and the one character after it
            const size_t at = (size_t)(k.p - lineBegin);
            std::string line(lineBegin, (size_t)(eol - lineBegin));
            if (!line.empty() && line.back() == '\r') line.pop_back();
            const size_t cut = at + 7 + 1;
            blk.comment = line.substr(0, at) + (cut < line.size() ? line.substr(cut) : std::string());
        }
        else if (k.is("lattice"))
        {
            if (blk.box.size() >= 9) throw std::runtime_error("ERROR: Too many box vectors.\n");
            for (size_t i = 1; i <= 3; ++i) blk.box.push_back(number(w, i));
        }
        else if (k.is("atom"))
        {
            if (w.size() < 10) throw std::out_of_range("ERROR: Atom line too short.\n");
            for (size_t i = 1; i <= 3; ++i) blk.pos.push_back(number(w, i));
            blk.el.push_back(w[4].str());
            blk.q.push_back(number(w, 5));
            for (size_t i = 7; i <= 9; ++i) blk.force.push_back(number(w, i));
        }
        else if (k.is("energy")) blk.energy = number(w, 1);
        else if (k.is("charge")) blk.charge = number(w, 1);
        else if (k.is("end"))
        {
            if (blk.box.size() != 0 && blk.box.size() != 9)
                throw std::runtime_error("ERROR: Strange number of box vectors.\n");
            commit(blk, out);
            inBlock = false;
        }
        else throw std::runtime_error("ERROR: Unexpected file content, unknown keyword \"" + k.str() + "\".\n");
    }
    return inBlock;
}

} // namespace

void readStructuresFile(std::string const& fileName, int64_t limit, StructureSet& out)
{
    std::FILE* f = std::fopen(fileName.c_str(), "rb");
    if (!f) throw std::runtime_error("ERROR: Could not open file: \"" + fileName + "\".\n");
    std::string text;
    char buf[1 << 16];
    if (std::fseek(f, 0, SEEK_END) == 0)
    {
        const long n = std::ftell(f);
        if (n > 0) text.reserve((size_t)n);
        std::fseek(f, 0, SEEK_SET);
    }
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, got);
    std::fclose(f);
    readStructures(text.c_str(), text.size(), limit, out);   // c_str(): NUL-terminated for strtod
}

} // namespace n2p2b200
