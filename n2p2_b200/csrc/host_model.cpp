// Host-side model setup; see host_model.hpp.  Reference citations are paths
// inside the n2p2 project.
#include "host_model.hpp"

#include <algorithm>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <sstream>
#include <stdexcept>

namespace n2p2b200 {

namespace {

std::string const kWhitespace = " \t";

std::string trimLine(std::string const& line)
{
    std::size_t b = line.find_first_not_of(kWhitespace);
    if (b == std::string::npos) return "";
    std::size_t e = line.find_last_not_of(kWhitespace);
    return line.substr(b, e - b + 1);
}

std::string fmt(char const* f, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof(buf), f, ap);
    va_end(ap);
    return buf;
}

// Keywords that may appear only once (Settings::sanityCheck, Settings.cpp:392-460).
bool repeatable(std::string const& key)
{
    return key == "symfunction" || key == "symfunction_short" || key == "atom_energy" ||
           key == "element_nodes_short" || key == "element_hidden_layers_short" ||
           key == "element_activation_short";
}

// Ordering of SymFnc*::operator< (SymFncExpRad.cpp:55-75,
// SymFncExpAngn.cpp:51-77, SymFncExpAngw.cpp:51-77): this order defines the
// index of every G in the network input.
bool sfLess(SymFunc const& a, SymFunc const& b)
{
    if (a.ec != b.ec) return a.ec < b.ec;
    if (a.type != b.type) return a.type < b.type;
    if (a.compact())
    {
        // SymFncCompRad / SymFncCompAngn / SymFncCompAngw::operator< (SymFncCompRad.cpp:50-66,
        // SymFncCompAngn.cpp:51-74, SymFncCompAngw.cpp:52-74); the weighted types have no
        // neighbour elements (SymFncCompRadWeighted.cpp:49-64, SymFncCompAngnWeighted.cpp:51-70,
        // SymFncCompAngwWeighted.cpp:51-70)
        if (a.subtype != b.subtype) return a.subtype < b.subtype;
        if (!a.weighted())
        {
            if (a.e1 != b.e1) return a.e1 < b.e1;
            if (!a.radial() && a.e2 != b.e2) return a.e2 < b.e2;
        }
        if (a.rc != b.rc) return a.rc < b.rc;
        if (a.rl != b.rl) return a.rl < b.rl;
        if (!a.radial())
        {
            if (a.angleLeft != b.angleLeft) return a.angleLeft < b.angleLeft;
            if (a.angleRight != b.angleRight) return a.angleRight < b.angleRight;
        }
        return false;
    }
    if (a.cutoffType != b.cutoffType) return a.cutoffType < b.cutoffType;
    if (a.cutoffAlpha != b.cutoffAlpha) return a.cutoffAlpha < b.cutoffAlpha;
    if (a.rc != b.rc) return a.rc < b.rc;
    if (a.eta != b.eta) return a.eta < b.eta;
    if (a.rs != b.rs) return a.rs < b.rs;
    if (a.type != 2)
    {
        if (a.zeta != b.zeta) return a.zeta < b.zeta;
        if (a.lambda != b.lambda) return a.lambda < b.lambda;
    }
    if (a.e1 != b.e1) return a.e1 < b.e1;
    if (a.type != 2 && a.e2 != b.e2) return a.e2 < b.e2;
    return false;
}

char const* const kKnownElements[] = {
    "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",
    "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn",
    "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh",
    "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd",
    "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",  "Re",
    "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th",
    "Pa", "U",  "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm", "Md", "No"};

} // namespace

std::string reduceLine(std::string const& line)
{
    std::string r = trimLine(line);
    std::string out;
    bool ws = false;
    for (char c : r)
    {
        if (c == ' ' || c == '\t')
        {
            ws = true;
            continue;
        }
        if (ws) out.push_back(' ');
        ws = false;
        out.push_back(c);
    }
    return out;
}

std::vector<std::string> splitWords(std::string const& line)
{
    std::vector<std::string> w;
    std::istringstream in(line);
    std::string s;
    while (in >> s) w.push_back(s);
    return w;
}

// --------------------------------------------------------------------------
// Settings
// --------------------------------------------------------------------------

void Settings::loadFile(std::string const& fileName)
{
    std::ifstream f(fileName);
    if (!f.is_open()) throw std::runtime_error("ERROR: Could not open file: \"" + fileName + "\".\n");
    std::stringstream ss;
    ss << f.rdbuf();
    parseText(ss.str());
}

void Settings::parseText(std::string const& text)
{
    contents_.clear();
    warnings_.clear();
    std::istringstream in(text);
    std::string line;
    std::size_t i = 0;
    for (; std::getline(in, line); ++i)
    {
        if (line.empty() || line == "\r") continue;
        std::size_t p = line.find('#');
        if (p != std::string::npos) line.erase(p);
        p = line.find('!');
        if (p != std::string::npos) line.erase(p);
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.find_first_not_of(' ') == std::string::npos) continue;
        line = reduceLine(line);
        if (line.empty()) continue;
        std::size_t sep = line.find(' ');
        if (sep == std::string::npos) contents_.insert({line, {"", i}});
        else contents_.insert({line.substr(0, sep), {line.substr(sep + 1), i}});
    }
    // Multiple instances of single-instance keywords are critical problems.
    std::size_t critical = 0;
    for (auto it = contents_.begin(); it != contents_.end(); it = contents_.upper_bound(it->first))
    {
        if (contents_.count(it->first) > 1 && !repeatable(it->first))
        {
            warnings_.push_back("WARNING (CRITICAL): Multiple instances of \"" + it->first + "\" detected.\n");
            critical++;
        }
    }
    if (critical > 0)
    {
        throw std::runtime_error(fmt("ERROR: %zu critical problem(s) were found in settings file.\n", critical));
    }
}

bool Settings::keywordExists(std::string const& key) const { return contents_.find(key) != contents_.end(); }

std::string const& Settings::value(std::string const& key) const
{
    auto it = contents_.find(key);
    if (it == contents_.end()) throw std::runtime_error("ERROR: Keyword \"" + key + "\" not found.\n");
    return it->second.first;
}

std::vector<std::pair<std::string, std::size_t>> Settings::values(std::string const& key) const
{
    std::vector<std::pair<std::string, std::size_t>> v;
    auto r = contents_.equal_range(key);
    for (auto it = r.first; it != r.second; ++it) v.push_back(it->second);
    return v;
}

// --------------------------------------------------------------------------
// Element map
// --------------------------------------------------------------------------

std::size_t ElementMap::atomicNumber(std::string const& symbol)
{
    std::size_t n = sizeof(kKnownElements) / sizeof(*kKnownElements);
    for (std::size_t i = 0; i < n; ++i)
        if (symbol == kKnownElements[i]) return i + 1;
    throw std::runtime_error("ERROR: Element \"" + symbol + "\" not found.\n");
}

int ElementMap::index(std::string const& symbol) const
{
    for (std::size_t i = 0; i < symbols.size(); ++i)
        if (symbols[i] == symbol) return (int)i;
    throw std::runtime_error("ERROR: Element \"" + symbol + "\" not in element map.\n");
}

int activationFromString(std::string const& c)
{
    // activationFromString (NeuralNetwork.cpp:1078-1098)
    if (c == "l") return AF_IDENTITY;
    if (c == "t") return AF_TANH;
    if (c == "s") return AF_LOGISTIC;
    if (c == "p") return AF_SOFTPLUS;
    if (c == "r") return AF_RELU;
    if (c == "g") return AF_GAUSSIAN;
    if (c == "c") return AF_COS;
    if (c == "S") return AF_REVLOGISTIC;
    if (c == "e") return AF_EXP;
    if (c == "h") return AF_HARMONIC;
    throw std::runtime_error("ERROR: Unknown activation function.\n");
}

// --------------------------------------------------------------------------
// SymFunc scaling (SymFnc::scale / unscale, SymFnc.cpp:169-223)
// --------------------------------------------------------------------------

double SymFunc::scale(double value) const
{
    switch (scalingType)
    {
    case ST_NONE: return value;
    case ST_SCALE: return Smin + scalingFactor * (value - Gmin);
    case ST_CENTER: return value - Gmean;
    case ST_SCALECENTER: return Smin + scalingFactor * (value - Gmean);
    case ST_SCALESIGMA: return Smin + scalingFactor * (value - Gmean);
    }
    return 0.0;
}

double SymFunc::unscale(double value) const
{
    switch (scalingType)
    {
    case ST_NONE: return value;
    case ST_SCALE: return (value - Smin) / scalingFactor + Gmin;
    case ST_CENTER: return value + Gmean;
    case ST_SCALECENTER: return (value - Smin) / scalingFactor + Gmean;
    case ST_SCALESIGMA: return (value - Smin) / scalingFactor + Gmean;
    }
    return 0.0;
}

// --------------------------------------------------------------------------
// Model setup
// --------------------------------------------------------------------------

void Model::loadSettingsFile(std::string const& fileName)
{
    settings.loadFile(fileName);
    loadSettingsText("");
}

void Model::loadSettingsText(std::string const& text)
{
    if (!text.empty()) settings.parseText(text);
    // Mode::loadSettingsFile: nnp_type selects the generation (Mode.cpp:177-205).
    if (settings.keywordExists("nnp_type"))
    {
        std::string t = settings.value("nnp_type");
        if (!(t == "2G-HDNNP" || t == "0"))
        {
            throw std::runtime_error("ERROR: Only short-range 2G-HDNNP models are supported (nnp_type \"" + t +
                                     "\").\n");
        }
    }
    setupDone = false;
    scalingDone = false;
}

void Model::setupGeneric()
{
    elements.clear();
    elementMap.symbols.clear();
    setupNormalization();
    setupElementMap();
    setupElements();
    setupCutoff();
    setupSymmetryFunctions();
    setupSymmetryFunctionMemory();
    setupSymmetryFunctionGroups();
    setupNeuralNetwork();
    setupDone = true;
}

void Model::setupNormalization()
{
    // Mode::setupNormalization (Mode.cpp:239-300)
    bool me = settings.keywordExists("mean_energy");
    bool ce = settings.keywordExists("conv_energy");
    bool cl = settings.keywordExists("conv_length");
    if (me && ce && cl)
    {
        normalize = true;
        meanEnergy = std::atof(settings.value("mean_energy").c_str());
        convEnergy = std::atof(settings.value("conv_energy").c_str());
        convLength = std::atof(settings.value("conv_length").c_str());
    }
    else if (!me && !ce && !cl && !settings.keywordExists("conv_charge"))
    {
        normalize = false;
        meanEnergy = 0.0;
        convEnergy = 1.0;
        convLength = 1.0;
    }
    else
    {
        throw std::runtime_error("ERROR: Incorrect usage of normalization keywords.\n"
                                 "       Use all or none of \"mean_energy\", \"conv_energy\" and \"conv_length\".\n");
    }
}

void Model::setupElementMap()
{
    // ElementMap::registerElements sorts by atomic number (ElementMap.cpp:40).
    std::vector<std::string> s = splitWords(settings.value("elements"));
    std::stable_sort(s.begin(), s.end(), [](std::string const& a, std::string const& b) {
        return ElementMap::atomicNumber(a) < ElementMap::atomicNumber(b);
    });
    if ((int)s.size() > kMaxElements) throw std::runtime_error("ERROR: Too many elements.\n");
    elementMap.symbols = s;
}

void Model::setupElements()
{
    // Mode::setupElements (Mode.cpp:323-367)
    std::size_t n = (std::size_t)std::atoi(settings.value("number_of_elements").c_str());
    if (n != elementMap.symbols.size()) throw std::runtime_error("ERROR: Inconsistent number of elements.\n");
    elements.resize(n);
    for (std::size_t i = 0; i < n; ++i)
    {
        elements[i].symbol = elementMap.symbols[i];
        elements[i].atomicNumber = ElementMap::atomicNumber(elementMap.symbols[i]);
    }
    for (auto const& v : settings.values("atom_energy"))
    {
        std::vector<std::string> a = splitWords(v.first);
        elements.at(elementMap.index(a.at(0))).atomicEnergyOffset = std::atof(a.at(1).c_str());
    }
}

void Model::setupCutoff()
{
    // Mode::setupCutoff (Mode.cpp:589-682)
    std::vector<std::string> a = splitWords(settings.value("cutoff_type"));
    cutoffType = std::atoi(a.at(0).c_str());
    cutoffAlpha = 0.0;
    if (a.size() > 1)
    {
        cutoffAlpha = std::atof(a.at(1).c_str());
        if (0.0 < cutoffAlpha && cutoffAlpha >= 1.0)
            throw std::invalid_argument("ERROR: 0 <= alpha < 1.0 is required.\n");
    }
    if (cutoffType < CT_HARD || cutoffType > CT_POLY4) throw std::invalid_argument("ERROR: Unknown cutoff type.\n");
}

void Model::setupSymmetryFunctions()
{
    // Mode::setupSymmetryFunctions (Mode.cpp:684-759) with
    // Element::addSymmetryFunction (Element.cpp:82-141) for types 2, 3, 9.
    for (auto const& v : settings.values("symfunction_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        SymFunc s;
        for (int e = 0; e < kMaxElements; ++e) s.indexPerElement[e] = -1;
        s.ec = elementMap.index(a.at(0));
        s.type = std::atoi(a.at(1).c_str());
        s.lineNumber = v.second;
        if (s.type == 2)
        {
            // SymFncExpRad::setParameters (SymFncExpRad.cpp:77-96)
            s.e1 = elementMap.index(a.at(2));
            s.eta = std::atof(a.at(3).c_str());
            s.rs = std::atof(a.at(4).c_str());
            s.rc = std::atof(a.at(5).c_str());
        }
        else if (s.type == 3 || s.type == 9)
        {
            // SymFncBaseExpAng::setParameters (SymFncBaseExpAng.cpp:50-93)
            s.e1 = elementMap.index(a.at(2));
            s.e2 = elementMap.index(a.at(3));
            s.eta = std::atof(a.at(4).c_str());
            s.lambda = std::atof(a.at(5).c_str());
            s.zeta = std::atof(a.at(6).c_str());
            s.rc = std::atof(a.at(7).c_str());
            if (a.size() > 8) s.rs = std::atof(a.at(8).c_str());
            if (s.e1 > s.e2) std::swap(s.e1, s.e2);
            s.zetaInt = (int)std::round(s.zeta);
            s.useIntegerPow = std::fabs(s.zeta - s.zetaInt) <= std::numeric_limits<double>::min();
        }
        else if (s.type >= 20 && s.type <= 25)
        {
            // SymFncCompRad::setParameters (SymFncCompRad.cpp:69-99),
            // SymFncBaseCompAng::setParameters (SymFncBaseCompAng.cpp:48-113),
            // SymFncCompRadWeighted::setParameters (SymFncCompRadWeighted.cpp:66-95),
            // SymFncBaseCompAngWeighted::setParameters (SymFncBaseCompAngWeighted.cpp:43-100)
            const bool rad = s.radial();
            const std::size_t ne = s.weighted() ? 0 : (rad ? 1 : 2);   // neighbour element fields
            if (ne > 0) s.e1 = elementMap.index(a.at(2));
            s.e2 = ne == 2 ? elementMap.index(a.at(3)) : s.e1;
            const std::size_t o = 2 + ne;
            s.rl = std::atof(a.at(o).c_str());
            s.rc = std::atof(a.at(o + 1).c_str());
            if (!rad)
            {
                s.angleLeft = std::atof(a.at(o + 2).c_str());
                s.angleRight = std::atof(a.at(o + 3).c_str());
            }
            s.subtype = a.at(o + (rad ? 2 : 4));
            if (!rad && s.e1 > s.e2) std::swap(s.e1, s.e2);
            if (s.rl > s.rc) throw std::runtime_error("ERROR: Lower radial boundary >= upper radial boundary.\n");
            // SymFncBaseComp::setCompactFunction (SymFncBaseComp.cpp:39-92)
            std::string const& t = s.subtype;
            if (t.size() < 1 || t.size() > 3)
                throw std::runtime_error("ERROR: Invalid compact function type specification: \"" + t + "\".\n");
            if (t.front() == 'p')
            {
                if (t.size() < 2) throw std::runtime_error("ERROR: Invalid polynom type: \"" + t + "\".\n");
                if (t[1] == '1') s.core = CORE_POLY1;
                else if (t[1] == '2') s.core = CORE_POLY2;
                else if (t[1] == '3') s.core = CORE_POLY3;
                else if (t[1] == '4') s.core = CORE_POLY4;
                else throw std::runtime_error("ERROR: Invalid polynom type: \"" + t + "\".\n");
                if (t.size() == 3)
                {
                    if (t[2] == 'a') s.asymmetric = true;
                    else throw std::runtime_error("ERROR: Invalid polynom specifier: \"" + t + "\".\n");
                }
            }
            else if (t.front() == 'e') s.core = CORE_EXP;
            else throw std::runtime_error("ERROR: Unknown compact SF type: \"" + t + "\".\n");
            if (!rad)
            {
                if (s.angleLeft >= s.angleRight)
                    throw std::runtime_error("ERROR: Left angle boundary right of or equal to right angle boundary.\n");
                const double center = (s.angleLeft + s.angleRight) / 2.0;
                if ((s.angleLeft < 0.0 && center != 0.0) || (s.angleRight > 180.0 && center != 180.0))
                    throw std::runtime_error("ERROR: Angle boundary out of [0,180] and center of angular function "
                                             "/= 0 or /= 180.\n");
                if (s.angleRight - s.angleLeft > 360.0)
                    throw std::runtime_error("ERROR: Periodic symmetry function cannot spread over domain > 360 "
                                             "degrees\n");
            }
        }
        else
        {
            throw std::runtime_error(fmt("ERROR: Symmetry function type %d is not supported by the GPU "
                                         "short-range path (supported: 2, 3, 9, 20-25).\n",
                                         s.type));
        }
        elements.at(s.ec).sf.push_back(s);
    }
    maxCutoffRadius = 0.0;
    for (auto& el : elements)
    {
        if (normalize)
        {
            // SymFncExpRad::changeLengthUnit / SymFncBaseExpAng::changeLengthUnit
            for (auto& s : el.sf)
            {
                s.eta /= convLength * convLength;
                s.rc *= convLength;
                s.rs *= convLength;
                s.rl *= convLength;   // compact: SymFncCompRad / SymFncBaseCompAng::changeLengthUnit
            }
        }
        // Element::sortSymmetryFunctions (Element.cpp:154-166)
        std::sort(el.sf.begin(), el.sf.end(), sfLess);
        for (std::size_t i = 0; i < el.sf.size(); ++i) el.sf[i].index = (int)i;
        for (auto& s : el.sf)
        {
            maxCutoffRadius = std::max(maxCutoffRadius, s.rc);
            s.cutoffType = cutoffType;
            s.cutoffAlpha = cutoffAlpha;
        }
        if (el.sf.empty()) throw std::runtime_error("ERROR: Element " + el.symbol + " has no symmetry functions.\n");
    }
}

void Model::setupSymmetryFunctionMemory()
{
    // Element::setupSymmetryFunctionMemory (Element.cpp:289-311)
    std::size_t ne = elements.size();
    for (auto& el : elements)
    {
        el.table.assign(ne, {});
        for (auto& s : el.sf)
        {
            for (std::size_t e = 0; e < ne; ++e)
            {
                if (s.relevant((int)e))
                {
                    s.indexPerElement[e] = (int)el.table[e].size();
                    el.table[e].push_back(s.index);
                }
            }
        }
    }
}

void Model::setupSymmetryFunctionGroups()
{
    // Element::setupSymmetryFunctionGroups (Element.cpp:194-287) and
    // SymGrp*::addMember / sortMembers (SymGrpExpRad.cpp:72-125,
    // SymGrpExpAngn.cpp:72-148).  The members are already in SF order, so
    // member order inside a group equals the reference's sorted member order.
    for (auto& el : elements)
    {
        el.groups.clear();
        el.compactGroups.clear();
        for (auto const& s : el.sf)
        {
            if (s.compact())
            {
                // SymGrpCompRad / SymGrpCompAngn / SymGrpCompAngw::operator== (SymGrpCompRad.cpp:39-46,
                // SymGrpCompAngn.cpp:36-44, SymGrpCompAngw.cpp:36-44): element pair only, any radii and
                // angles; the weighted groups take every member of their type
                // (SymGrpCompRadWeighted.cpp:37-42, SymGrpCompAngwWeighted.cpp:36-41)
                SymGroup* cg = nullptr;
                for (auto& cand : el.compactGroups)
                    if (cand.type == s.type &&
                        (s.weighted() || (cand.e1 == s.e1 && (s.radial() || cand.e2 == s.e2))))
                        cg = &cand;
                if (!cg)
                {
                    el.compactGroups.emplace_back();
                    cg = &el.compactGroups.back();
                    cg->type = s.type;
                    cg->ec = s.ec;
                    cg->e1 = s.e1;
                    cg->e2 = s.e2;
                }
                // calculateComp: the first member and every member whose radial boundaries differ
                // from its predecessor's (SymGrpCompAngn.cpp:110-126, SymGrpCompAngnWeighted.cpp:98-114)
                const bool comp = cg->members.empty() || el.sf[cg->members.back()].rc != s.rc ||
                                  el.sf[cg->members.back()].rl != s.rl;
                cg->rc = std::max(cg->rc, s.rc);
                cg->members.push_back(s.index);
                cg->calculateComp.push_back(comp ? 1 : 0);
                continue;
            }
            SymGroup* g = nullptr;
            for (auto& cand : el.groups)
            {
                if (cand.type == s.type && cand.cutoffType == s.cutoffType && cand.cutoffAlpha == s.cutoffAlpha &&
                    cand.ec == s.ec && cand.rc == s.rc && cand.e1 == s.e1 && (s.type == 2 || cand.e2 == s.e2))
                {
                    g = &cand;
                    break;
                }
            }
            if (!g)
            {
                el.groups.emplace_back();
                g = &el.groups.back();
                g->type = s.type;
                g->ec = s.ec;
                g->e1 = s.e1;
                g->e2 = s.e2;
                g->rc = s.rc;
                g->cutoffType = s.cutoffType;
                g->cutoffAlpha = s.cutoffAlpha;
            }
            g->members.push_back(s.index);
        }
        for (auto& g : el.groups)
        {
            g.calculateExp.clear();
            g.factorNorm.clear();
            g.factorDeriv.clear();
            for (std::size_t m = 0; m < g.members.size(); ++m)
            {
                SymFunc const& s = el.sf[g.members[m]];
                if (g.type != 2)
                {
                    g.factorNorm.push_back(std::pow(2.0, 1.0 - s.zeta));
                    g.factorDeriv.push_back(2.0 * s.eta / s.zeta / s.lambda);
                }
                bool ce = true;
                if (m > 0)
                {
                    SymFunc const& p = el.sf[g.members[m - 1]];
                    ce = (p.eta != s.eta || p.rs != s.rs);
                }
                g.calculateExp.push_back(ce ? 1 : 0);
            }
        }
    }
}

void Model::setupNeuralNetwork()
{
    // Mode::setupNeuralNetwork (Mode.cpp:1227-1512), short-range network only.
    std::size_t ne = elements.size();
    std::size_t globalHidden = 0;
    std::vector<NetworkTopology> topo(ne);
    if (settings.keywordExists("global_hidden_layers_short"))
    {
        globalHidden = (std::size_t)std::atoi(settings.value("global_hidden_layers_short").c_str());
        for (auto& t : topo) t.numLayers = (int)globalHidden + 2;
    }
    for (auto const& v : settings.values("element_hidden_layers_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        topo.at(elementMap.index(a.at(0))).numLayers = std::atoi(a.at(1).c_str()) + 2;
    }
    for (auto& t : topo)
    {
        if (t.numLayers == 0) throw std::runtime_error("ERROR: Number of neural network hidden layers unset for some elements.\n");
        t.neurons.assign(t.numLayers, 0);
        t.activations.assign(t.numLayers, AF_UNSET);
    }
    std::vector<std::string> gNodes, gAct;
    if (settings.keywordExists("global_nodes_short"))
    {
        gNodes = splitWords(settings.value("global_nodes_short"));
        if (globalHidden != gNodes.size())
            throw std::runtime_error("ERROR: Inconsistent global NN topology keyword \"global_nodes_short\".\n");
    }
    if (settings.keywordExists("global_activation_short"))
    {
        gAct = splitWords(settings.value("global_activation_short"));
        if (globalHidden != gAct.size() - 1)
            throw std::runtime_error("ERROR: Inconsistent global NN topology keyword \"global_activation_short\".\n");
    }
    for (std::size_t i = 0; i < ne; ++i)
    {
        NetworkTopology& t = topo[i];
        t.neurons[0] = (int)elements[i].sf.size();
        t.activations[0] = AF_IDENTITY;
        t.neurons[t.numLayers - 1] = 1;
        if ((std::size_t)t.numLayers != globalHidden + 2) continue;
        for (int j = 1; j < t.numLayers; ++j)
        {
            if (j == t.numLayers - 1 && !gAct.empty())
            {
                t.activations[j] = activationFromString(gAct.at(t.numLayers - 2));
            }
            else
            {
                if (!gNodes.empty()) t.neurons[j] = std::atoi(gNodes.at(j - 1).c_str());
                if (!gAct.empty()) t.activations[j] = activationFromString(gAct.at(j - 1));
            }
        }
    }
    // Per-element overrides; the index ranges follow the reference
    // (Mode.cpp:1400-1440) exactly.
    for (auto const& v : settings.values("element_nodes_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        NetworkTopology& t = topo.at(elementMap.index(a.at(0)));
        std::size_t n = a.size() - 1;
        if ((std::size_t)t.numLayers != n + 2)
            throw std::runtime_error("ERROR: Inconsistent per-element NN topology keyword \"element_nodes_short\".\n");
        for (int j = 1; j < t.numLayers - 2; ++j) t.neurons[j] = std::atoi(a.at(j).c_str());
    }
    for (auto const& v : settings.values("element_activation_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        NetworkTopology& t = topo.at(elementMap.index(a.at(0)));
        std::size_t n = a.size() - 1;
        if ((std::size_t)t.numLayers != n + 1)
            throw std::runtime_error("ERROR: Inconsistent per-element NN topology keyword \"element_activation_short\".\n");
        for (int j = 1; j < t.numLayers - 1; ++j) t.activations[j] = activationFromString(a.at(j));
    }
    for (std::size_t i = 0; i < ne; ++i)
    {
        for (int j = 0; j < topo[i].numLayers; ++j)
        {
            if (topo[i].neurons[j] == 0)
                throw std::runtime_error(fmt("ERROR: NN \"short\", element %2s: number of neurons for layer %d unset.\n",
                                             elements[i].symbol.c_str(), j));
            if (topo[i].activations[j] == AF_UNSET)
                throw std::runtime_error(fmt("ERROR: NN \"short\", element %2s: activation functions for layer %d unset.\n",
                                             elements[i].symbol.c_str(), j));
        }
        if (topo[i].numLayers < 3) throw std::runtime_error("ERROR: Neural network must have at least three layers\n");
        elements[i].topology = topo[i];
        elements[i].hasWeights = false;
        elements[i].W.assign(topo[i].numLayers - 1, {});
        elements[i].b.assign(topo[i].numLayers - 1, {});
    }
    normalizeNeurons = settings.keywordExists("normalize_nodes");
}

void Model::setupSymmetryFunctionScalingNone()
{
    // Element::setScalingNone (Element.cpp:338-357)
    for (auto& el : elements)
    {
        for (auto& s : el.sf)
        {
            s.scalingType = ST_NONE;
            s.Gmin = s.Gmax = s.Gmean = s.Gsigma = 0.0;
            s.Smin = s.Smax = 0.0;
            s.scalingFactor = 1.0;
        }
        for (auto& g : el.groups)
        {
            if (g.type == 2) continue;
            for (std::size_t m = 0; m < g.members.size(); ++m)
                g.factorNorm[m] = std::pow(2.0, 1.0 - el.sf[g.members[m]].zeta) * el.sf[g.members[m]].scalingFactor;
        }
    }
    scalingType = ST_NONE;
    scalingDone = true;
}

void Model::setupSymmetryFunctionScaling(std::string const& fileName)
{
    // Mode::setupSymmetryFunctionScaling (Mode.cpp:781-909)
    bool sc = settings.keywordExists("scale_symmetry_functions");
    bool ce = settings.keywordExists("center_symmetry_functions");
    if (sc && !ce) scalingType = ST_SCALE;
    else if (!sc && ce) scalingType = ST_CENTER;
    else if (sc && ce) scalingType = ST_SCALECENTER;
    else if (settings.keywordExists("scale_symmetry_functions_sigma")) scalingType = ST_SCALESIGMA;
    else scalingType = ST_NONE;

    double Smin = 0.0, Smax = 0.0;
    if (scalingType == ST_SCALE || scalingType == ST_SCALECENTER || scalingType == ST_SCALESIGMA)
    {
        Smin = settings.keywordExists("scale_min_short") ? std::atof(settings.value("scale_min_short").c_str()) : 0.0;
        Smax = settings.keywordExists("scale_max_short") ? std::atof(settings.value("scale_max_short").c_str()) : 1.0;
    }

    std::ifstream file(fileName);
    if (!file.is_open()) throw std::runtime_error("ERROR: Could not open file: \"" + fileName + "\".\n");
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(file, line))
    {
        if (line.empty()) continue;
        if (line.at(0) != '#') lines.push_back(line);
    }
    std::size_t pos = 0;
    for (auto& el : elements)
    {
        for (auto& s : el.sf)
        {
            if (pos >= lines.size()) throw std::runtime_error("ERROR: Too few lines in scaling file.\n");
            std::vector<std::string> w = splitWords(lines[pos++]);
            // SymFnc::setScalingType (SymFnc.cpp:52-98)
            if (((std::size_t)std::atoi(w.at(0).c_str()) != (std::size_t)s.ec + 1) &&
                ((std::size_t)std::atoi(w.at(1).c_str()) != (std::size_t)s.index + 1))
            {
                throw std::runtime_error("ERROR: Inconsistent scaling statistics.\n");
            }
            s.scalingType = scalingType;
            s.Gmin = std::atof(w.at(2).c_str());
            s.Gmax = std::atof(w.at(3).c_str());
            s.Gmean = std::atof(w.at(4).c_str());
            if (w.size() > 5) s.Gsigma = std::atof(w.at(5).c_str());
            s.Smin = Smin;
            s.Smax = Smax;
            switch (scalingType)
            {
            case ST_NONE: s.scalingFactor = 1.0; break;
            case ST_SCALE: s.scalingFactor = (Smax - Smin) / (s.Gmax - s.Gmin); break;
            case ST_CENTER: s.scalingFactor = 1.0; break;
            case ST_SCALECENTER: s.scalingFactor = (Smax - Smin) / (s.Gmax - s.Gmin); break;
            case ST_SCALESIGMA: s.scalingFactor = (Smax - Smin) / s.Gsigma; break;
            }
        }
        // SymGrpBaseExpAng::setScalingFactors (SymGrpBaseExpAng.cpp:45-57)
        for (auto& g : el.groups)
        {
            if (g.type == 2) continue;
            for (std::size_t m = 0; m < g.members.size(); ++m)
                g.factorNorm[m] = std::pow(2.0, 1.0 - el.sf[g.members[m]].zeta) * el.sf[g.members[m]].scalingFactor;
        }
    }
    scalingDone = true;
}

void Model::setConnections(int element, std::vector<double> const& c)
{
    // NeuralNetwork::setConnections (NeuralNetwork.cpp:147-169): per layer,
    // for each source neuron j, for each target k: w(k <- j); then biases.
    ElementSetup& el = elements.at(element);
    NetworkTopology const& t = el.topology;
    std::size_t need = 0;
    for (int l = 1; l < t.numLayers; ++l) need += (std::size_t)t.neurons[l] * t.neurons[l - 1] + t.neurons[l];
    if (c.size() < need)
        throw std::runtime_error(fmt("ERROR: Element %s: %zu weights given, %zu required.\n", el.symbol.c_str(),
                                     c.size(), need));
    std::size_t count = 0;
    for (int l = 1; l < t.numLayers; ++l)
    {
        int nin = t.neurons[l - 1], nout = t.neurons[l];
        el.W[l - 1].assign((std::size_t)nin * nout, 0.0);
        el.b[l - 1].assign(nout, 0.0);
        for (int j = 0; j < nin; ++j)
            for (int k = 0; k < nout; ++k) el.W[l - 1][(std::size_t)k * nin + j] = c[count++];
        for (int k = 0; k < nout; ++k) el.b[l - 1][k] = c[count++];
    }
    el.hasWeights = true;
}

void Model::setupNeuralNetworkWeights(std::string const& fileNameFormat)
{
    // Mode::readNeuralNetworkWeights (Mode.cpp:2331-2350) with
    // readColumnsFromFile (utility.cpp:247-290), first column, '#' comments.
    for (std::size_t i = 0; i < elements.size(); ++i)
    {
        char name[4096];
        snprintf(name, sizeof(name), fileNameFormat.c_str(), elements[i].atomicNumber);
        std::ifstream f(name);
        if (!f.is_open()) throw std::runtime_error(std::string("ERROR: Could not open file: \"") + name + "\".\n");
        std::vector<double> c;
        std::string line;
        while (std::getline(f, line))
        {
            if (line.empty() || line.at(0) == '#') continue;
            std::vector<std::string> w = splitWords(line);
            c.push_back(w.empty() ? std::numeric_limits<double>::quiet_NaN() : std::atof(w[0].c_str()));
        }
        setConnections((int)i, c);
    }
}

} // namespace n2p2b200
