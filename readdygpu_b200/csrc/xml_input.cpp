// xml_input.cpp -- Xerces-free reader of the ReaDDy input files and the
// C API of include/readdy_b200_inputs.h.
#include <map>
#include "xml_input.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "readdy_b200_inputs.h"

namespace rdxml {

const Node* Node::child(const std::string& n) const
{
    for (auto& k : kids)
        if (k->name == n) return k.get();
    return nullptr;
}

std::vector<const Node*> Node::children(const std::string& n) const
{
    std::vector<const Node*> v;
    for (auto& k : kids)
        if (k->name == n) v.push_back(k.get());
    return v;
}

std::string trim(const std::string& s)
{
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

std::string Node::child_text(const std::string& n, const std::string& dflt) const
{
    const Node* c = child(n);
    return c ? trim(c->text) : dflt;
}

bool read_file(const std::string& path, std::string& out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

namespace {
std::string decode(const std::string& s)
{
    std::string o;
    for (size_t i = 0; i < s.size(); ++i) {
        if (s[i] == '&') {
            size_t e = s.find(';', i);
            if (e != std::string::npos) {
                std::string ent = s.substr(i + 1, e - i - 1);
                const char* rep = ent == "lt" ? "<" : ent == "gt" ? ">" : ent == "amp" ? "&" : ent == "quot" ? "\"" : ent == "apos" ? "'" : nullptr;
                if (rep) { o += rep; i = e; continue; }
            }
        }
        o += s[i];
    }
    return o;
}
}  // namespace

std::unique_ptr<Node> parse(const std::string& src, std::string& err)
{
    std::vector<Node*> stack;
    std::unique_ptr<Node> root;
    size_t i = 0, n = src.size();
    while (i < n) {
        if (src[i] != '<') {
            size_t j = src.find('<', i);
            if (j == std::string::npos) j = n;
            if (!stack.empty()) stack.back()->text += decode(src.substr(i, j - i));
            i = j;
            continue;
        }
        if (src.compare(i, 4, "<!--") == 0) {
            size_t j = src.find("-->", i + 4);
            if (j == std::string::npos) { err = "unterminated comment"; return nullptr; }
            i = j + 3;
            continue;
        }
        if (src.compare(i, 2, "<?") == 0 || src.compare(i, 2, "<!") == 0) {
            size_t j = src.find('>', i);
            if (j == std::string::npos) { err = "unterminated declaration"; return nullptr; }
            i = j + 1;
            continue;
        }
        if (src.compare(i, 2, "</") == 0) {
            size_t j = src.find('>', i);
            if (j == std::string::npos) { err = "unterminated end tag"; return nullptr; }
            std::string nm = trim(src.substr(i + 2, j - i - 2));
            if (stack.empty() || stack.back()->name != nm) { err = "mismatched end tag </" + nm + ">"; return nullptr; }
            stack.pop_back();
            i = j + 1;
            continue;
        }
        // start tag
        size_t j = i + 1;
        while (j < n && !isspace((unsigned char)src[j]) && src[j] != '>' && src[j] != '/') ++j;
        auto node = std::make_unique<Node>();
        node->name = src.substr(i + 1, j - i - 1);
        bool selfclose = false;
        while (j < n) {
            while (j < n && isspace((unsigned char)src[j])) ++j;
            if (j < n && src[j] == '>') { ++j; break; }
            if (j + 1 < n && src[j] == '/' && src[j + 1] == '>') { selfclose = true; j += 2; break; }
            size_t k = j;
            while (k < n && src[k] != '=' && !isspace((unsigned char)src[k]) && src[k] != '>') ++k;
            std::string an = src.substr(j, k - j);
            while (k < n && isspace((unsigned char)src[k])) ++k;
            if (k >= n || src[k] != '=') { err = "attribute without value in <" + node->name + ">"; return nullptr; }
            ++k;
            while (k < n && isspace((unsigned char)src[k])) ++k;
            if (k >= n || (src[k] != '"' && src[k] != '\'')) { err = "unquoted attribute in <" + node->name + ">"; return nullptr; }
            char q = src[k];
            size_t e = src.find(q, k + 1);
            if (e == std::string::npos) { err = "unterminated attribute"; return nullptr; }
            node->attrs[an] = decode(src.substr(k + 1, e - k - 1));
            j = e + 1;
        }
        Node* raw = node.get();
        if (stack.empty()) {
            if (root) { err = "more than one root element"; return nullptr; }
            root = std::move(node);
        } else {
            stack.back()->kids.push_back(std::move(node));
        }
        if (!selfclose) stack.push_back(raw);
        i = j;
    }
    if (!stack.empty()) { err = "unclosed element <" + stack.back()->name + ">"; return nullptr; }
    if (!root) { err = "no root element"; return nullptr; }
    return root;
}

}  // namespace rdxml

// ===========================================================================
// ReaDDy input files -> rdgpu_system_desc
// ===========================================================================
struct rdgpu_inputs {
    rdgpu_system_desc desc;
    rdgpu_run_params run;
    std::vector<double> xyz;
    std::vector<int32_t> types, ids;
    std::string error;
    // particle groups as bonds: gpu indices, potential index, potentials
    std::vector<int32_t> bond_ij, bond_pot;
    std::vector<rdgpu_pair_pot> bond_pots;
    int32_t groups_unsupported = 0;
};

namespace {
thread_local std::string g_err;

std::vector<double> numbers(const std::string& s)
{
    std::vector<double> v;
    const char* p = s.c_str();
    while (*p) {
        if (strchr("+-0123456789.", *p)) {
            char* e;
            double d = strtod(p, &e);
            if (e != p) { v.push_back(d); p = e; continue; }
        }
        ++p;
    }
    return v;
}

// "[0,1]" / "all" / "" (Simulation.cpp:65-77 parseAffectedIds)
std::vector<int> type_list(const std::string& s, int S)
{
    std::vector<int> v;
    std::string t = rdxml::trim(s);
    if (t == "all") { for (int i = 0; i < S; ++i) v.push_back(i); return v; }
    if (t == "null") return v;
    for (double d : numbers(t)) v.push_back((int)d);
    return v;
}

// "[[1,1];[0,1]]" / "all" (Simulation.cpp:78-92 parse2AffectedIds)
std::vector<std::pair<int, int>> pair_list(const std::string& s, int S)
{
    std::vector<std::pair<int, int>> v;
    std::string t = rdxml::trim(s);
    if (t == "all") {
        for (int i = 0; i < S; ++i)
            for (int j = 0; j < S; ++j) v.push_back({i, j});
        return v;
    }
    if (t == "null") return v;
    std::vector<double> d = numbers(t);
    for (size_t k = 0; k + 1 < d.size(); k += 2) v.push_back({(int)d[k], (int)d[k + 1]});
    return v;
}

int subtype_of(const std::string& s)
{
    if (s == "attractive") return RDGPU_SUB_ATTRACTIVE;
    if (s == "repulsive") return RDGPU_SUB_REPULSIVE;
    if (s == "spring") return RDGPU_SUB_SPRING;
    if (s == "membrane") return RDGPU_SUB_MEMBRANE;
    return 0;
}

bool load(const char* path, std::unique_ptr<rdxml::Node>& root, std::string& err)
{
    std::string src;
    if (!path || !*path || !rdxml::read_file(path, src)) { err = std::string("cannot read ") + (path ? path : "(null)"); return false; }
    std::string e;
    root = rdxml::parse(src, e);
    if (!root) { err = std::string(path) + ": " + e; return false; }
    return true;
}

int read_all(rdgpu_inputs* I, const char* pp, const char* tp, const char* pg, const char* tc, double max_cutoff)
{
    rdgpu_system_desc& d = I->desc;
    memset(&d, 0, sizeof(d));
    memset(&I->run, 0, sizeof(I->run));
    const int M = RDGPU_MAX_TYPES;
    // ---- param_particles.xml (ParticleParametersHandler.cpp:111-160)
    std::unique_ptr<rdxml::Node> root;
    if (!load(pp, root, I->error)) return RDGPU_ERR_ARG;
    auto parts = root->children("particle");
    if (parts.empty() || (int)parts.size() > M) { I->error = "param_particles: 1..16 <particle> entries needed"; return RDGPU_ERR_ARG; }
    d.n_types = (int)parts.size();
    std::map<std::string, int> type_id;
    for (int t = 0; t < d.n_types; ++t) type_id[parts[t]->child_text("type")] = t;
    for (int t = 0; t < d.n_types; ++t) {
        const rdxml::Node* p = parts[t];
        d.D[t] = atof(p->child_text("diffusionConstant", "0").c_str());
        double dflt = 0.0;
        std::map<int, double> spec;
        if (const rdxml::Node* cm = p->child("collisionRadiusMap")) {
            for (const rdxml::Node* cr : cm->children("collisionRadius")) {
                std::string partners = cr->child_text("partnerType");
                double r = atof(cr->child_text("radius", "0").c_str());
                std::stringstream ss(partners);
                std::string nm;
                while (std::getline(ss, nm, ',')) {
                    nm = rdxml::trim(nm);
                    if (nm == "default" || nm == "all") dflt = r;
                    else if (type_id.count(nm)) spec[type_id[nm]] = r;
                }
            }
        }
        d.p_radius[t] = dflt;
        for (int j = 0; j < d.n_types; ++j) d.coll_radius[t * M + j] = spec.count(j) ? spec[j] : dflt;
    }
    // ---- tplgy_potentials.xml (PotentialParametersHandler.cpp:51-79, Simulation.cpp:230-251)
    if (!load(tp, root, I->error)) return RDGPU_ERR_ARG;
    for (const rdxml::Node* p : root->children("pot")) {
        auto at = [&](const char* k, const char* dflt = "") {
            auto it = p->attrs.find(k);
            return it == p->attrs.end() ? std::string(dflt) : it->second;
        };
        std::string type = at("type");
        int sub = subtype_of(at("subtype"));
        if (type == "HARMONIC" || type == "WEAK_INTERACTION_PIECEWISE_HARMONIC") {
            if (rdxml::trim(at("affectedParticleIdPairs")) != "" && rdxml::trim(at("affectedParticleIdPairs")) != "null")
                I->run.n_unsupported++;
            auto prs = pair_list(at("affectedParticleTypeIdPairs"), d.n_types);
            if (prs.empty()) continue;
            if (d.n_pair >= RDGPU_MAX_PAIR_POTS) { I->error = "too many pair potentials"; return RDGPU_ERR_ARG; }
            rdgpu_pair_pot& q = d.pair[d.n_pair++];
            q.kind = type == "HARMONIC" ? RDGPU_P2_HARMONIC : RDGPU_P2_WEAK_PIECEWISE;
            q.subtype = q.kind == RDGPU_P2_HARMONIC ? sub : 0;
            q.k = atof(at("forceConst", "0").c_str());
            std::string r0 = rdxml::trim(at("r0", "null"));
            q.r0 = (r0.empty() || r0 == "null") ? -1.0 : atof(r0.c_str());
            q.length = atof(at("length", "0").c_str());
            q.depth = atof(at("depth", "0").c_str());
            for (auto& pr : prs) {
                if (pr.first < 0 || pr.first >= d.n_types || pr.second < 0 || pr.second >= d.n_types) continue;
                q.pairs[pr.first * M + pr.second] = 1;
                q.pairs[pr.second * M + pr.first] = 1;
            }
        } else if (type == "DISK" || type == "CYLINDER" || type == "SPHERE" || type == "CUBE" || type == "BOX") {
            auto tl = type_list(at("affectedParticleTypeIds"), d.n_types);
            if (tl.empty()) continue;
            if (d.n_ext >= RDGPU_MAX_EXT_POTS) { I->error = "too many external potentials"; return RDGPU_ERR_ARG; }
            rdgpu_ext_pot& q = d.ext[d.n_ext++];
            q.kind = type == "DISK" ? RDGPU_P1_DISK : type == "CYLINDER" ? RDGPU_P1_CYLINDER
                   : type == "SPHERE" ? RDGPU_P1_SPHERE : RDGPU_P1_CUBE;
            q.subtype = sub;
            q.k = atof(at("forceConst", "0").c_str());
            auto c = numbers(at("center", "[0,0,0]"));
            auto nn = numbers(at("normal", "[0,0,1]"));
            auto o = numbers(at("origin", "[0,0,0]"));
            auto e = numbers(at("extension", "[0,0,0]"));
            for (int a = 0; a < 3; ++a) {
                q.center[a] = a < (int)c.size() ? c[a] : 0.0;
                q.normal[a] = a < (int)nn.size() ? nn[a] : 0.0;
                q.origin[a] = a < (int)o.size() ? o[a] : 0.0;
                q.extension[a] = a < (int)e.size() ? e[a] : 0.0;
            }
            q.radius = atof(at("radius", "0").c_str());
            q.height = atof(at("height", "0").c_str());
            q.consider_radius = rdxml::trim(at("considerParticleRadius", "true")) != "false";
            for (int t : tl)
                if (t >= 0 && t < d.n_types) q.types[t] = 1;
        } else if (type == "WEAK_INTERACTION_HARMONIC" || type == "WEAK_INTERACTION") {
            // the cubic weak interaction (the reference GPU's
            // CudaSimulation.cu:1021-1031, Java's P2_WeakInteraction) is not
            // implemented here: refuse the input rather than run without it
            I->error = "pair potential type " + type + " (cubic weak interaction) is not supported by this core; "
                       "use WEAK_INTERACTION_PIECEWISE_HARMONIC";
            return RDGPU_ERR_ARG;
        } else {
            I->run.n_unsupported++;   // types neither the reference's GPU core nor this one knows
        }
    }
    // ---- param_global.xml (GlobalParametersHandler.cpp:73-143, XMLReader.cpp:67)
    if (!load(pg, root, I->error)) return RDGPU_ERR_ARG;
    double dt_frame = atof(root->child_text("dt", "0").c_str());
    double dt = 0.0;
    for (const char* k : {"dtOpenMM", "dt_dynamic", "dt_dyn"})
        if (root->child(k)) dt = atof(root->child_text(k).c_str());
    if (!(dt > 0)) dt = dt_frame;
    I->run.dt_frame = dt_frame;
    I->run.n_frames = atoll(root->child_text("nSimulationSteps", "0").c_str());
    I->run.steps_per_frame = dt > 0 ? (int64_t)std::llround(dt_frame / dt) : 1;
    if (I->run.steps_per_frame < 1) I->run.steps_per_frame = 1;
    std::string dev = root->child_text("cudaDeviceIndex", root->child_text("cudaDevice", "0"));
    I->run.device = atoi(dev.c_str());
    I->run.testmode = atoi(root->child_text("testmode", "0").c_str()) == 1;
    d.dt = dt;
    d.T = atof(root->child_text("T", "0").c_str());
    d.kB = atof(root->child_text("Kb", "0.0083144621").c_str());
    auto lb = numbers(root->child_text("latticeBounds", ""));
    if (lb.size() != 6) { I->error = "param_global: latticeBounds needs [[x0,x1];[y0,y1];[z0,z1]]"; return RDGPU_ERR_ARG; }
    for (int a = 0; a < 3; ++a) {
        d.lo[a] = lb[2 * a];
        d.hi[a] = lb[2 * a + 1];
        d.periodic[a] = 1;   // the GPU core is periodic in all axes (CudaSimulation.cu:1857-1858)
    }
    d.max_cutoff = max_cutoff;
    // ---- tplgy_coordinates.xml (CoordReader.cpp:16-65); a trajectory written
    // by rdgpu_traj_write (<traj> of frames) restarts from its last frame
    if (!load(tc, root, I->error)) return RDGPU_ERR_ARG;
    const rdxml::Node* coords = root.get();
    if (root->name == "traj") {
        auto frames = root->children("tplgy_coords");
        if (frames.empty()) { I->error = "tplgy_coordinates: <traj> without a <tplgy_coords> frame"; return RDGPU_ERR_ARG; }
        coords = frames.back();
    }
    for (const rdxml::Node* p : coords->children("p")) {
        auto c = numbers(p->attrs.count("c") ? p->attrs.at("c") : "");
        if (c.size() != 3 || !p->attrs.count("type")) { I->error = "tplgy_coordinates: bad <p> entry"; return RDGPU_ERR_ARG; }
        I->ids.push_back(p->attrs.count("id") ? atoi(p->attrs.at("id").c_str()) : (int)I->ids.size());
        I->types.push_back(atoi(p->attrs.at("type").c_str()));
        for (int a = 0; a < 3; ++a) I->xyz.push_back(c[a]);
    }
    return RDGPU_OK;
}
// param_groups.xml / tplgy_groups.xml (GroupParametersHandler.cpp:41-190,
// GroupReader.cpp:13-40): group type k is the k-th <particleGroup>; each of
// its HARMONIC / WEAK_INTERACTION_PIECEWISE_HARMONIC potentials acts on the
// internal-id pairs it names; a <g type="k" internalAndParticleId="[[u,id];...]">
// instance maps internal ids to ReaDDy particle ids.
int read_groups(rdgpu_inputs* I, const char* pgr, const char* tgr)
{
    I->bond_ij.clear();
    I->bond_pot.clear();
    I->bond_pots.clear();
    I->groups_unsupported = 0;
    std::unique_ptr<rdxml::Node> root;
    if (!load(pgr, root, I->error)) return RDGPU_ERR_ARG;
    struct GroupPot { int index; std::vector<std::pair<int, int>> pairs; };
    std::vector<std::vector<GroupPot>> gtypes;
    for (const rdxml::Node* g : root->children("particleGroup")) {
        std::vector<GroupPot> gp;
        if (const rdxml::Node* ps = g->child("potentials")) {
            for (const rdxml::Node* p : ps->children("pot")) {
                auto at = [&](const char* kk, const char* dflt = "") {
                    auto it = p->attrs.find(kk);
                    return it == p->attrs.end() ? std::string(dflt) : it->second;
                };
                const std::string type = at("type");
                if (type != "HARMONIC" && type != "WEAK_INTERACTION_PIECEWISE_HARMONIC") {
                    I->groups_unsupported++;   // e.g. StiffnessInteraction
                    continue;
                }
                rdgpu_pair_pot q;
                memset(&q, 0, sizeof(q));
                q.kind = type == "HARMONIC" ? RDGPU_P2_HARMONIC : RDGPU_P2_WEAK_PIECEWISE;
                q.subtype = q.kind == RDGPU_P2_HARMONIC ? subtype_of(at("subtype")) : 0;
                if (q.kind == RDGPU_P2_HARMONIC && q.subtype == 0) { I->error = "param_groups: harmonic subtype missing"; return RDGPU_ERR_ARG; }
                q.k = atof(at("forceConst", "0").c_str());
                const std::string r0 = rdxml::trim(at("r0", "null"));
                q.r0 = (r0.empty() || r0 == "null") ? -1.0 : atof(r0.c_str());
                q.length = atof(at("length", "0").c_str());
                q.depth = atof(at("depth", "0").c_str());
                I->bond_pots.push_back(q);
                std::vector<std::pair<int, int>> prs;
                std::vector<double> v = numbers(at("affectedInternalIdPairs"));
                for (size_t t = 0; t + 1 < v.size(); t += 2) prs.push_back({(int)v[t], (int)v[t + 1]});
                gp.push_back({(int)I->bond_pots.size() - 1, prs});
            }
        }
        gtypes.push_back(gp);
    }
    if (!load(tgr, root, I->error)) return RDGPU_ERR_ARG;
    std::map<int, int> index_of;   // ReaDDy particle id -> gpu index
    for (size_t i = 0; i < I->ids.size(); ++i) index_of[I->ids[i]] = (int)i;
    for (const rdxml::Node* g : root->children("g")) {
        auto it = g->attrs.find("type");
        auto ip = g->attrs.find("internalAndParticleId");
        if (it == g->attrs.end() || ip == g->attrs.end()) { I->error = "tplgy_groups: <g> needs type and internalAndParticleId"; return RDGPU_ERR_ARG; }
        const int gt = atoi(it->second.c_str());
        if (gt < 0 || gt >= (int)gtypes.size()) { I->error = "tplgy_groups: group type out of range"; return RDGPU_ERR_ARG; }
        std::map<int, int> part;
        std::vector<double> v = numbers(ip->second);
        for (size_t t = 0; t + 1 < v.size(); t += 2) {
            auto f = index_of.find((int)v[t + 1]);
            if (f == index_of.end()) { I->error = "tplgy_groups: unknown particle id " + std::to_string((int)v[t + 1]); return RDGPU_ERR_ARG; }
            part[(int)v[t]] = f->second;
        }
        for (const GroupPot& p : gtypes[gt])
            for (auto& pr : p.pairs) {
                if (!part.count(pr.first) || !part.count(pr.second)) { I->error = "tplgy_groups: internal id missing from a group instance"; return RDGPU_ERR_ARG; }
                I->bond_ij.push_back(part[pr.first]);
                I->bond_ij.push_back(part[pr.second]);
                I->bond_pot.push_back(p.index);
            }
    }
    return RDGPU_OK;
}
}  // namespace

extern "C" {

int rdgpu_inputs_read_groups(rdgpu_inputs_handle h, const char* param_groups, const char* tplgy_groups)
{
    if (!h) return RDGPU_ERR_ARG;
    return read_groups(h, param_groups, tplgy_groups);
}

int rdgpu_inputs_bond_counts(rdgpu_inputs_handle h, int64_t* n_bonds, int32_t* n_pots, int32_t* n_unsupported)
{
    if (!h) return RDGPU_ERR_ARG;
    if (n_bonds) *n_bonds = (int64_t)h->bond_pot.size();
    if (n_pots) *n_pots = (int32_t)h->bond_pots.size();
    if (n_unsupported) *n_unsupported = h->groups_unsupported;
    return RDGPU_OK;
}

int rdgpu_inputs_bonds(rdgpu_inputs_handle h, int32_t* ij, int32_t* pot, rdgpu_pair_pot* pots)
{
    if (!h) return RDGPU_ERR_ARG;
    if (ij) memcpy(ij, h->bond_ij.data(), h->bond_ij.size() * sizeof(int32_t));
    if (pot) memcpy(pot, h->bond_pot.data(), h->bond_pot.size() * sizeof(int32_t));
    if (pots) memcpy(pots, h->bond_pots.data(), h->bond_pots.size() * sizeof(rdgpu_pair_pot));
    return RDGPU_OK;
}

int rdgpu_inputs_read(const char* param_particles, const char* tplgy_potentials, const char* param_global,
                      const char* tplgy_coordinates, double max_cutoff, rdgpu_inputs_handle* out)
{
    if (!out) return RDGPU_ERR_ARG;
    auto* I = new rdgpu_inputs();
    int rc = read_all(I, param_particles, tplgy_potentials, param_global, tplgy_coordinates, max_cutoff);
    if (rc) {
        g_err = I->error;
        delete I;
        *out = nullptr;
        return rc;
    }
    *out = I;
    return RDGPU_OK;
}

int rdgpu_inputs_desc(rdgpu_inputs_handle h, rdgpu_system_desc* desc, rdgpu_run_params* run)
{
    if (!h) return RDGPU_ERR_ARG;
    if (desc) *desc = h->desc;
    if (run) *run = h->run;
    return RDGPU_OK;
}

int64_t rdgpu_inputs_count(rdgpu_inputs_handle h) { return h ? (int64_t)h->types.size() : 0; }

int rdgpu_inputs_particles(rdgpu_inputs_handle h, double* xyz, int32_t* types, int32_t* ids)
{
    if (!h) return RDGPU_ERR_ARG;
    if (xyz) memcpy(xyz, h->xyz.data(), h->xyz.size() * sizeof(double));
    if (types) memcpy(types, h->types.data(), h->types.size() * sizeof(int32_t));
    if (ids) memcpy(ids, h->ids.data(), h->ids.size() * sizeof(int32_t));
    return RDGPU_OK;
}

const char* rdgpu_inputs_error(rdgpu_inputs_handle h) { return h ? h->error.c_str() : g_err.c_str(); }

void rdgpu_inputs_free(rdgpu_inputs_handle h) { delete h; }

}  // extern "C"
