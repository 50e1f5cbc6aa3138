// Input and output formats of the reference launcher, rewritten for this library:
//   - the XML tissue model (ParseInputFile, base/xmcml/xmcmlLauncher/parser.cpp:18-514),
//   - the binary .surface file (ParseSurfaceFile, parser.cpp:516-611):
//       u32 0x0100 | i32 nSurf | { i32 nV | nV x 3 f64 | i32 nT | nT x 3 i32 } x nSurf
//   - the sectioned binary .mcml.out (WriteOutputToFile, writer.cpp:431-471; section ids
//     sections.h:4-19), each section [u32 id][u32 length][payload],
//   - InitOutput / FreeOutput (launcher_omp.cpp:10-58, 76-104).
// The XML reader is a small recursive-descent parser of elements and text written here (the
// reference uses tinyxml); field names, defaults and the detector re-ordering are the reference's.
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "xmc_internal.h"

namespace xmc {
namespace {

struct XNode {
    std::string name;
    std::string text;
    std::vector<std::unique_ptr<XNode>> kids;
};

class XmlReader {
  public:
    explicit XmlReader(const std::string& s) : s_(s) {}

    std::unique_ptr<XNode> parse(std::string* err) {
        skip_misc();
        auto root = element(err, 0);
        return root;
    }

  private:
    const std::string& s_;
    size_t i_ = 0;

    bool starts(const char* p) const { return s_.compare(i_, std::strlen(p), p) == 0; }
    void skip_ws() { while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_; }
    void skip_misc() {
        for (;;) {
            skip_ws();
            if (starts("<?")) { size_t e = s_.find("?>", i_); i_ = e == std::string::npos ? s_.size() : e + 2; }
            else if (starts("<!--")) { size_t e = s_.find("-->", i_); i_ = e == std::string::npos ? s_.size() : e + 3; }
            else if (starts("<!")) { size_t e = s_.find('>', i_); i_ = e == std::string::npos ? s_.size() : e + 1; }
            else break;
        }
    }
    static std::string unescape(const std::string& t) {
        std::string o;
        for (size_t k = 0; k < t.size(); ++k) {
            if (t[k] == '&') {
                size_t e = t.find(';', k);
                if (e != std::string::npos) {
                    std::string ent = t.substr(k + 1, e - k - 1);
                    if (ent == "lt") { o += '<'; k = e; continue; }
                    if (ent == "gt") { o += '>'; k = e; continue; }
                    if (ent == "amp") { o += '&'; k = e; continue; }
                    if (ent == "quot") { o += '"'; k = e; continue; }
                    if (ent == "apos") { o += '\''; k = e; continue; }
                }
            }
            o += t[k];
        }
        return o;
    }
    std::unique_ptr<XNode> element(std::string* err, int depth) {
        if (depth > 64) { *err = "XML nested too deeply"; return nullptr; }
        if (i_ >= s_.size() || s_[i_] != '<') { *err = "XML: expected an element"; return nullptr; }
        ++i_;
        size_t b = i_;
        while (i_ < s_.size() && !std::isspace((unsigned char)s_[i_]) && s_[i_] != '>' && s_[i_] != '/') ++i_;
        auto n = std::make_unique<XNode>();
        n->name = s_.substr(b, i_ - b);
        if (n->name.empty()) { *err = "XML: empty element name"; return nullptr; }
        // attributes are ignored (the reference's format has none)
        while (i_ < s_.size() && s_[i_] != '>' && !(s_[i_] == '/' && i_ + 1 < s_.size() && s_[i_ + 1] == '>')) {
            if (s_[i_] == '"' || s_[i_] == '\'') { char q = s_[i_++]; while (i_ < s_.size() && s_[i_] != q) ++i_; }
            ++i_;
        }
        if (i_ >= s_.size()) { *err = "XML: unterminated tag <" + n->name + ">"; return nullptr; }
        if (s_[i_] == '/') { i_ += 2; return n; }
        ++i_;
        std::string text;
        for (;;) {
            if (i_ >= s_.size()) { *err = "XML: missing </" + n->name + ">"; return nullptr; }
            if (starts("<!--")) { size_t e = s_.find("-->", i_); i_ = e == std::string::npos ? s_.size() : e + 3; continue; }
            if (starts("<![CDATA[")) {
                size_t e = s_.find("]]>", i_);
                if (e == std::string::npos) { *err = "XML: unterminated CDATA"; return nullptr; }
                text += s_.substr(i_ + 9, e - i_ - 9);
                i_ = e + 3;
                continue;
            }
            if (starts("</")) {
                i_ += 2;
                size_t b2 = i_;
                while (i_ < s_.size() && s_[i_] != '>') ++i_;
                std::string close = s_.substr(b2, i_ - b2);
                while (!close.empty() && std::isspace((unsigned char)close.back())) close.pop_back();
                if (close != n->name) { *err = "XML: </" + close + "> closes <" + n->name + ">"; return nullptr; }
                ++i_;
                break;
            }
            if (s_[i_] == '<') {
                auto k = element(err, depth + 1);
                if (!k) return nullptr;
                n->kids.push_back(std::move(k));
                continue;
            }
            text += s_[i_++];
        }
        size_t a = text.find_first_not_of(" \t\r\n"), z = text.find_last_not_of(" \t\r\n");
        n->text = a == std::string::npos ? std::string() : unescape(text.substr(a, z - a + 1));
        return n;
    }
};

double xf(const XNode* n) { return std::atof(n->text.c_str()); }
int xi(const XNode* n) { return std::atoi(n->text.c_str()); }

void read_xyz(const XNode* n, xmc_ref_double3* v, bool as_int) {
    for (auto& k : n->kids) {
        double val = as_int ? (double)xi(k.get()) : xf(k.get());
        if (k->name == "X") v->x = val;
        else if (k->name == "Y") v->y = val;
        else if (k->name == "Z") v->z = val;
    }
}

template <class D>
bool read_filter(const XNode* n, D* d, int* count, std::string* err) {
    for (int j = 0; j < MAX_LAYERS; ++j) d->filterLayers[j] = false;
    *count = 0;
    for (auto& k : n->kids) {
        if (k->name != "Layer") continue;
        int l = xi(k.get());
        if (l < 0 || l >= MAX_LAYERS) { *err = "FilterLayers invalid"; return false; }
        d->filterLayers[l] = true;
        ++*count;
    }
    return true;
}

bool parse_input(const char* path, InputInfo* in, std::string* err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { *err = std::string("cannot open ") + path; return false; }
    std::stringstream ss;
    ss << f.rdbuf();
    std::string s = ss.str();
    XmlReader rd(s);
    auto root = rd.parse(err);
    if (!root) return false;

    // defaults: parser.cpp:20-48
    std::memset(in, 0, sizeof(*in));
    in->timeScaleSize = 1;
    in->startDirection.z = 1.0;
    in->weightIntegralPrecision = 128;
    in->weightTablePrecision = 262144;
    in->attractiveFactor = 1.0;

    const XNode* layers = nullptr;
    const XNode* cubes = nullptr;
    const XNode* rings = nullptr;
    for (auto& kp : root->kids) {
        const XNode* k = kp.get();
        const std::string& nm = k->name;
        if (nm == "NumberOfPhotons") in->numberOfPhotons = std::strtoull(k->text.c_str(), nullptr, 10);
        else if (nm == "MinWeight") in->minWeight = xf(k);
        else if (nm == "TimeStart") in->timeStart = xf(k);
        else if (nm == "TimeFinish") in->timeFinish = xf(k);
        else if (nm == "TimeScaleSize") in->timeScaleSize = xi(k);
        else if (nm == "TargetRange") {
            for (auto& c : k->kids)
                if (c->name == "Layer") {
                    int l = xi(c.get());
                    if (l >= 0 && l < MAX_LAYERS) in->targetRangeLayers[l] = 1;
                }
        } else if (nm == "StartPosition") read_xyz(k, &in->startPosition, false);
        else if (nm == "StartDirection") read_xyz(k, &in->startDirection, false);
        else if (nm == "Area") {
            if (!in->area) { in->area = new Area; std::memset(in->area, 0, sizeof(Area)); }
            for (auto& c : k->kids) {
                if (c->name == "Corner") read_xyz(c.get(), &in->area->corner, false);
                else if (c->name == "Length") read_xyz(c.get(), &in->area->length, false);
                else if (c->name == "PartitionNumber") {
                    xmc_ref_double3 p{};
                    read_xyz(c.get(), &p, true);
                    in->area->partitionNumber.x = (int)p.x;
                    in->area->partitionNumber.y = (int)p.y;
                    in->area->partitionNumber.z = (int)p.z;
                }
            }
        } else if (nm == "Biasing") {
            in->useBiasing = 1;
            for (auto& c : k->kids) {
                if (c->name == "WeightIntegral") {
                    for (auto& w : c->kids) {
                        if (w->name == "IntegralPrecision") in->weightIntegralPrecision = (uint)xi(w.get());
                        if (w->name == "TablePrecision") in->weightTablePrecision = (uint)xi(w.get());
                        if (w->name == "AttractiveFactor") in->attractiveFactor = xf(w.get());
                    }
                } else if (c->name == "TargetPoint") {
                    read_xyz(c.get(), &in->targetPoint, true);  // atoi, as parser.cpp:233-241
                }
            }
        } else if (nm == "NumberOfLayers") in->numberOfLayers = xi(k);
        else if (nm == "Layers") layers = k;
        else if (nm == "NumberOfCubeDetectors") in->numberOfCubeDetectors = xi(k);
        else if (nm == "CubeDetectors") cubes = k;
        else if (nm == "NumberOfRingDetectors") in->numberOfRingDetectors = xi(k);
        else if (nm == "RingDetectors") rings = k;
        else if (nm == "NumberOfSurfaces") in->numberOfSurfaces = xi(k);
    }
    if (in->numberOfLayers <= 0) { *err = "NumberOfLayers missing"; return false; }
    in->layerInfo = new LayerInfo[in->numberOfLayers];
    std::memset(in->layerInfo, 0, sizeof(LayerInfo) * in->numberOfLayers);
    if (layers) {
        int i = 0;
        for (auto& lp : layers->kids) {
            if (i >= in->numberOfLayers) { *err = "number of layers invalid"; return false; }
            if (lp->name == "Layer") {
                LayerInfo& L = in->layerInfo[i];
                const XNode* ids = nullptr;
                for (auto& c : lp->kids) {
                    if (c->name == "RefractiveIndex") L.refractiveIndex = xf(c.get());
                    else if (c->name == "AbsorptionCoefficient") L.absorptionCoefficient = xf(c.get());
                    else if (c->name == "ScatteringCoefficient") L.scatteringCoefficient = xf(c.get());
                    else if (c->name == "Anisotropy") L.anisotropy = xf(c.get());
                    else if (c->name == "NumberOfSurfaces") L.numberOfSurfaces = xi(c.get());
                    else if (c->name == "SurfaceIds") ids = c.get();
                }
                if (ids) {
                    L.surfaceId = new int[std::max(1, L.numberOfSurfaces)];
                    int j = 0;
                    for (auto& c : ids->kids) {
                        if (c->name != "Id") { ++j; continue; }
                        if (j >= L.numberOfSurfaces) { *err = "layer surface ids exceed NumberOfSurfaces"; return false; }
                        L.surfaceId[j++] = xi(c.get());
                    }
                } else if (L.numberOfSurfaces > 0) {
                    *err = "layer lists NumberOfSurfaces but no SurfaceIds";
                    return false;
                }
            }
            ++i;
        }
    }
    // Detectors are kept in a stable order by their number of filter layers: the reference
    // stores them in std::multimap<int, ...> keyed by that count (parser.cpp:59-60,488,498-511).
    auto sort_by_filters = [](auto& v) {
        std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    };
    if (in->numberOfCubeDetectors > 0) {
        std::vector<std::pair<int, CubeDetector>> v;
        if (cubes) {
            int i = 0;
            for (auto& dp : cubes->kids) {
                if (i >= in->numberOfCubeDetectors) { *err = "number of cube detectors invalid"; return false; }
                ++i;
                if (dp->name != "CubeDetector") continue;
                CubeDetector d;
                std::memset(&d, 0, sizeof(d));
                for (int j = 0; j < MAX_LAYERS; ++j) d.filterLayers[j] = true;
                int nf = MAX_LAYERS;
                d.targetAngle = 90.0;
                for (auto& c : dp->kids) {
                    if (c->name == "Center") read_xyz(c.get(), &d.center, false);
                    else if (c->name == "Length") read_xyz(c.get(), &d.length, false);
                    else if (c->name == "Filter") { if (!read_filter(c.get(), &d, &nf, err)) return false; }
                    else if (c->name == "TargetAngle") d.targetAngle = xf(c.get());
                }
                v.push_back({nf, d});
            }
        }
        if ((int)v.size() != in->numberOfCubeDetectors) { *err = "number of cube detectors invalid"; return false; }
        sort_by_filters(v);
        in->cubeDetector = new CubeDetector[v.size()];
        for (size_t i = 0; i < v.size(); ++i) in->cubeDetector[i] = v[i].second;
    }
    if (in->numberOfRingDetectors > 0) {
        std::vector<std::pair<int, RingDetector>> v;
        if (rings) {
            int i = 0;
            for (auto& dp : rings->kids) {
                if (i >= in->numberOfRingDetectors) { *err = "number of ring detectors invalid"; return false; }
                ++i;
                if (dp->name != "RingDetector") continue;
                RingDetector d;
                std::memset(&d, 0, sizeof(d));
                for (int j = 0; j < MAX_LAYERS; ++j) d.filterLayers[j] = true;
                int nf = MAX_LAYERS;
                d.targetAngle = 90.0;
                for (auto& c : dp->kids) {
                    if (c->name == "Center") read_xyz(c.get(), &d.center, false);
                    else if (c->name == "SmallRadius") d.smallRadius = xf(c.get());
                    else if (c->name == "BigRadius") d.bigRadius = xf(c.get());
                    else if (c->name == "Filter") { if (!read_filter(c.get(), &d, &nf, err)) return false; }
                    else if (c->name == "TargetAngle") d.targetAngle = xf(c.get());
                }
                v.push_back({nf, d});
            }
        }
        if ((int)v.size() != in->numberOfRingDetectors) { *err = "number of ring detectors invalid"; return false; }
        sort_by_filters(v);
        in->ringDetector = new RingDetector[v.size()];
        for (size_t i = 0; i < v.size(); ++i) in->ringDetector[i] = v[i].second;
    }
    if (!in->area) { *err = "Area missing"; return false; }
    return true;
}

bool parse_surface(const char* path, InputInfo* in, std::string* err) {
    FILE* f = std::fopen(path, "rb");
    if (!f) { *err = std::string("cannot open ") + path; return false; }
    std::unique_ptr<FILE, int (*)(FILE*)> guard(f, std::fclose);
    uint32_t id = 0;
    int32_t ns = 0;
    if (std::fread(&id, 4, 1, f) != 1 || id != 0x0100u) { *err = "not a .surface file (section id)"; return false; }
    if (std::fread(&ns, 4, 1, f) != 1 || ns != in->numberOfSurfaces) { *err = "surface count differs from NumberOfSurfaces"; return false; }
    if (ns < 0) { *err = "negative surface count"; return false; }
    in->surface = new Surface[ns > 0 ? ns : 1];
    std::memset(in->surface, 0, sizeof(Surface) * (ns > 0 ? ns : 1));
    for (int s = 0; s < ns; ++s) {
        Surface& S = in->surface[s];
        int32_t nv = 0, nt = 0;
        if (std::fread(&nv, 4, 1, f) != 1 || nv < 0) { *err = "truncated .surface file (vertex count)"; return false; }
        S.numberOfVertices = nv;
        S.vertices = new xmc_ref_double3[nv > 0 ? nv : 1];
        if (nv > 0 && std::fread(S.vertices, sizeof(xmc_ref_double3), (size_t)nv, f) != (size_t)nv) { *err = "truncated .surface file (vertices)"; return false; }
        if (std::fread(&nt, 4, 1, f) != 1 || nt < 0) { *err = "truncated .surface file (triangle count)"; return false; }
        S.numberOfTriangles = nt;
        S.triangles = new xmc_ref_int3[nt > 0 ? nt : 1];
        if (nt > 0 && std::fread(S.triangles, sizeof(xmc_ref_int3), (size_t)nt, f) != (size_t)nt) { *err = "truncated .surface file (triangles)"; return false; }
    }
    return true;
}

struct Writer {
    FILE* f;
    bool ok = true;
    template <class T>
    void put(const T& v) { ok = ok && std::fwrite(&v, sizeof(T), 1, f) == 1; }
    void put_n(const void* p, size_t size, size_t n) { ok = ok && (n == 0 || std::fwrite(p, size, n, f) == n); }
    void section(uint32_t id, uint32_t len) { put(id); put(len); }
};

}  // namespace
}  // namespace xmc

using namespace xmc;

extern "C" {

bool xmc_parse_input_file(const char* fileName, InputInfo* input) {
    std::string err;
    if (!fileName || !input) { set_error("NULL argument"); return false; }
    bool ok = parse_input(fileName, input, &err);
    if (!ok) set_error("ParseInputFile: " + err);
    return ok;
}

bool xmc_parse_surface_file(const char* fileName, InputInfo* input) {
    std::string err;
    if (!fileName || !input) { set_error("NULL argument"); return false; }
    bool ok = parse_surface(fileName, input, &err);
    if (!ok) set_error("ParseSurfaceFile: " + err);
    return ok;
}

void xmc_free_input(InputInfo* in) {
    if (!in) return;
    delete in->area;
    if (in->layerInfo) {
        for (int i = 0; i < in->numberOfLayers; ++i) delete[] in->layerInfo[i].surfaceId;
        delete[] in->layerInfo;
    }
    if (in->surface) {
        for (int s = 0; s < in->numberOfSurfaces; ++s) {
            delete[] in->surface[s].vertices;
            delete[] in->surface[s].triangles;
        }
        delete[] in->surface;
    }
    delete[] in->cubeDetector;
    delete[] in->ringDetector;
    if (in->weightTable) {
        for (int k = 0; k < in->numberOfWeightTables; ++k) delete[] in->weightTable[k].elements;
        delete[] in->weightTable;
    }
    std::memset(in, 0, sizeof(*in));
}

// launcher_omp.cpp:10-58
void xmc_init_output(InputInfo* in, OutputInfo* out) {
    out->numberOfPhotons = 0;
    out->specularReflectance = 0.0;
    const int grid = in->area->partitionNumber.x * in->area->partitionNumber.y * in->area->partitionNumber.z;
    out->gridSize = grid;
    out->absorption = new double[grid]();
    out->scattering = new double[grid]();
    const int nd = in->numberOfCubeDetectors + in->numberOfRingDetectors;
    out->numberOfDetectors = nd;
    out->detectorInfo = new DetectorInfo[nd > 0 ? nd : 1];
    const int T = in->timeScaleSize;
    double step = (in->timeFinish - in->timeStart) / T;
    if (step < 0.0) step = 0.0;
    for (int i = 0; i < nd; ++i) {
        DetectorInfo& D = out->detectorInfo[i];
        D.weight = 0;
        D.numberOfPhotons = 0;
        D.trajectorySize = grid;
        D.trajectory = new uint64[grid]();
        D.timeScaleSize = T;
        D.timeScale = new TimeInfo[T]();
        for (int j = 0; j < T - 1; ++j) {
            D.timeScale[j].timeStart = in->timeStart + j * step;
            D.timeScale[j].timeFinish = D.timeScale[j].timeStart + step;
        }
        D.timeScale[T - 1].timeStart = in->timeStart + (T - 1) * step;
        D.timeScale[T - 1].timeFinish = in->timeFinish;
        D.targetWeight = 0.0;
    }
}

// launcher_omp.cpp:76-104
void xmc_free_output(OutputInfo* out) {
    if (!out) return;
    delete[] out->absorption;
    delete[] out->scattering;
    if (out->detectorInfo) {
        for (int i = 0; i < out->numberOfDetectors; ++i) {
            delete[] out->detectorInfo[i].trajectory;
            delete[] out->detectorInfo[i].timeScale;
        }
        delete[] out->detectorInfo;
    }
    std::memset(out, 0, sizeof(*out));
}

// writer.cpp:431-471 with the section layouts of writer.cpp:32-429
bool xmc_write_output_file(InputInfo* in, OutputInfo* out, const char* fileName) {
    FILE* f = std::fopen(fileName, "wb");
    if (!f) { set_error(std::string("cannot open ") + fileName); return false; }
    Writer w{f};
    const int nc = in->numberOfCubeDetectors, nr = in->numberOfRingDetectors, nd = out->numberOfDetectors;
    const int grid = out->gridSize;
    w.section(0x01, sizeof(uint64));                                   // number of photons
    w.put((uint64)in->numberOfPhotons);
    w.section(0x02, 6 * sizeof(double) + 3 * sizeof(int));             // area
    const Area& a = *in->area;
    double ad[6] = {a.corner.x, a.corner.y, a.corner.z, a.length.x, a.length.y, a.length.z};
    int ai[3] = {a.partitionNumber.x, a.partitionNumber.y, a.partitionNumber.z};
    w.put_n(ad, sizeof(double), 6);
    w.put_n(ai, sizeof(int), 3);
    w.section(0x03, (uint32_t)(sizeof(int) + 6 * sizeof(double) * nc));  // cube detectors
    w.put(nc);
    for (int i = 0; i < nc; ++i) {
        const CubeDetector& d = in->cubeDetector[i];
        double b[6] = {d.center.x, d.center.y, d.center.z, d.length.x, d.length.y, d.length.z};
        w.put_n(b, sizeof(double), 6);
    }
    w.section(0x0A, (uint32_t)(sizeof(int) + 5 * sizeof(double) * nr));  // ring detectors
    w.put(nr);
    for (int i = 0; i < nr; ++i) {
        const RingDetector& d = in->ringDetector[i];
        double b[5] = {d.center.x, d.center.y, d.center.z, d.smallRadius, d.bigRadius};
        w.put_n(b, sizeof(double), 5);
    }
    w.section(0x04, sizeof(double));                                   // specular reflectance
    w.put(out->specularReflectance);
    w.section(0x05, (uint32_t)(sizeof(int) + grid * sizeof(double)));  // absorption
    w.put(grid);
    w.put_n(out->absorption, sizeof(double), grid);
    w.section(0x0C, (uint32_t)(sizeof(int) + grid * sizeof(double)));  // scattering
    w.put(grid);
    w.put_n(out->scattering, sizeof(double), grid);
    w.section(0x06, (uint32_t)(sizeof(int) + nd * sizeof(double)));    // detector weights
    w.put(nd);
    for (int i = 0; i < nd; ++i) w.put(out->detectorInfo[i].weight);
    uint32_t len = sizeof(int);                                        // detector trajectories
    for (int i = 0; i < nd; ++i) len += sizeof(uint64) + sizeof(int) + out->detectorInfo[i].trajectorySize * sizeof(uint64);
    w.section(0x07, len);
    w.put(nd);
    for (int i = 0; i < nd; ++i) {
        const DetectorInfo& D = out->detectorInfo[i];
        w.put(D.numberOfPhotons);
        w.put(D.trajectorySize);
        w.put_n(D.trajectory, sizeof(uint64), D.trajectorySize);
    }
    len = sizeof(int);                                                 // time scales
    for (int i = 0; i < nd; ++i) len += sizeof(int) + out->detectorInfo[i].timeScaleSize * (4 * sizeof(double) + sizeof(uint64));
    w.section(0x08, len);
    w.put(nd);
    for (int i = 0; i < nd; ++i) {
        const DetectorInfo& D = out->detectorInfo[i];
        w.put(D.timeScaleSize);
        for (int j = 0; j < D.timeScaleSize; ++j) {
            w.put(D.timeScale[j].timeStart);
            w.put(D.timeScale[j].timeFinish);
            w.put(D.timeScale[j].numberOfPhotons);
            w.put(D.timeScale[j].weight);
            w.put(D.timeScale[j].targetWeight);
        }
    }
    w.section(0x0B, (uint32_t)(sizeof(int) + 2 * nd * sizeof(double)));  // detector ranges
    w.put(nd);
    for (int i = 0; i < nd; ++i) {
        const DetectorInfo& D = out->detectorInfo[i];
        w.put(D.weight - D.targetWeight);
        w.put(D.targetWeight);
    }
    std::fflush(f);
    bool ok = w.ok && std::fclose(f) == 0;
    if (!ok) set_error(std::string("write failed: ") + fileName);
    return ok;
}

int xmc_layout_offsets(int64_t* o, int max_count) {
    int64_t v[] = {
        (int64_t)sizeof(xmc_ref_double3), (int64_t)sizeof(xmc_ref_int3), (int64_t)sizeof(byte3),
        (int64_t)sizeof(Area), (int64_t)offsetof(Area, length), (int64_t)offsetof(Area, partitionNumber),
        (int64_t)sizeof(Surface), (int64_t)offsetof(Surface, numberOfVertices), (int64_t)offsetof(Surface, triangles),
        (int64_t)offsetof(Surface, numberOfTriangles),
        (int64_t)sizeof(BVHNode), (int64_t)offsetof(BVHNode, rightNode), (int64_t)offsetof(BVHNode, leftNode),
        (int64_t)offsetof(BVHNode, offset), (int64_t)offsetof(BVHNode, numOfTriangles),
        (int64_t)sizeof(BVHTree), (int64_t)offsetof(BVHTree, numOfNodes), (int64_t)offsetof(BVHTree, root),
        (int64_t)offsetof(BVHTree, triangles), (int64_t)offsetof(BVHTree, numOfTriangles),
        (int64_t)sizeof(Triangle),
        (int64_t)sizeof(TimeInfo), (int64_t)offsetof(TimeInfo, numberOfPhotons), (int64_t)offsetof(TimeInfo, weight),
        (int64_t)offsetof(TimeInfo, targetWeight),
        (int64_t)sizeof(CubeDetector), (int64_t)offsetof(CubeDetector, length), (int64_t)offsetof(CubeDetector, filterLayers),
        (int64_t)offsetof(CubeDetector, targetAngle),
        (int64_t)sizeof(RingDetector), (int64_t)offsetof(RingDetector, smallRadius), (int64_t)offsetof(RingDetector, bigRadius),
        (int64_t)offsetof(RingDetector, filterLayers), (int64_t)offsetof(RingDetector, targetAngle),
        (int64_t)sizeof(DetectorInfo), (int64_t)offsetof(DetectorInfo, trajectory), (int64_t)offsetof(DetectorInfo, trajectorySize),
        (int64_t)offsetof(DetectorInfo, timeScale), (int64_t)offsetof(DetectorInfo, timeScaleSize),
        (int64_t)offsetof(DetectorInfo, targetWeight), (int64_t)offsetof(DetectorInfo, weight),
        (int64_t)sizeof(WeightIntegralTable), (int64_t)offsetof(WeightIntegralTable, numberOfElements),
        (int64_t)offsetof(WeightIntegralTable, elements),
        (int64_t)sizeof(LayerInfo), (int64_t)offsetof(LayerInfo, absorptionCoefficient),
        (int64_t)offsetof(LayerInfo, scatteringCoefficient), (int64_t)offsetof(LayerInfo, anisotropy),
        (int64_t)offsetof(LayerInfo, surfaceId), (int64_t)offsetof(LayerInfo, numberOfSurfaces),
        (int64_t)sizeof(InputInfo), (int64_t)offsetof(InputInfo, area), (int64_t)offsetof(InputInfo, layerInfo),
        (int64_t)offsetof(InputInfo, numberOfLayers), (int64_t)offsetof(InputInfo, surface),
        (int64_t)offsetof(InputInfo, numberOfSurfaces), (int64_t)offsetof(InputInfo, cubeDetector),
        (int64_t)offsetof(InputInfo, numberOfCubeDetectors), (int64_t)offsetof(InputInfo, ringDetector),
        (int64_t)offsetof(InputInfo, numberOfRingDetectors), (int64_t)offsetof(InputInfo, minWeight),
        (int64_t)offsetof(InputInfo, bvhTree), (int64_t)offsetof(InputInfo, timeStart), (int64_t)offsetof(InputInfo, timeFinish),
        (int64_t)offsetof(InputInfo, timeScaleSize), (int64_t)offsetof(InputInfo, startPosition),
        (int64_t)offsetof(InputInfo, startDirection), (int64_t)offsetof(InputInfo, useBiasing),
        (int64_t)offsetof(InputInfo, weightIntegralPrecision), (int64_t)offsetof(InputInfo, weightTablePrecision),
        (int64_t)offsetof(InputInfo, attractiveFactor), (int64_t)offsetof(InputInfo, weightTable),
        (int64_t)offsetof(InputInfo, numberOfWeightTables), (int64_t)offsetof(InputInfo, targetPoint),
        (int64_t)offsetof(InputInfo, targetRangeLayers),
        (int64_t)sizeof(OutputInfo), (int64_t)offsetof(OutputInfo, specularReflectance), (int64_t)offsetof(OutputInfo, absorption),
        (int64_t)offsetof(OutputInfo, scattering), (int64_t)offsetof(OutputInfo, gridSize),
        (int64_t)offsetof(OutputInfo, detectorInfo), (int64_t)offsetof(OutputInfo, numberOfDetectors),
        (int64_t)sizeof(MCG59), (int64_t)offsetof(MCG59, offset),
    };
    int n = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < max_count; ++i) o[i] = v[i];
    return n;
}

}  // extern "C"
