// Host-side scene loading: pine's scene-file grammar and factories, flattened into the
// pg_scene_desc arrays that pg_upload_scene takes.
//
//   Parse / ParseBlock        src/util/parser.cpp:9-110
//   Parameters                src/util/parameters.h:13-89, parameters.cpp:20-163
//   pstd::stof/stoi/stofs     src/pstd/string.cpp:37-120
//   LoadObj                   src/util/objloader.cpp:12-100
//   LoadVolume                src/util/fileio.cpp:194-202
//   LoadScene                 src/util/fileio.cpp:251-281
//   Create{Material,BSDF,Node,Medium,Light,Shape,Camera,Film,Integrator}
//                             material.cpp:65-82, bxdf.cpp:170-196, node.cpp:33-97,
//                             medium.cpp:190-224, light.cpp:141-182, geometry.cpp:323-411,
//                             camera.cpp:9-14,86-107, film.cpp:7-12, integrator.cpp:20-56
//
// Unknown types follow pine: a warning and pine's fallback, except where pine's fallback
// is a component this library does not implement (texture nodes, Cylinder/Disk/Line,
// Atmosphere, emissive meshes), which fail with PG_ERR_UNSUPPORTED.
#include "scene_load.h"

#include <algorithm>
#include <iterator>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>

#include "pg_math.h"
#include "pg_nodes.h"

namespace pg {

// ---------------------------------------------------------------- pstd string parsing
static bool IsNumber(char c) {
    return c >= '0' && c <= '9';
}
static bool IsSpace(char c) {
    return c == ' ' || c == '\n' || c == '\t' || c == '\r' || c == '\f';
}

// pstd::stof (string.cpp:50-68): a digit accumulator, no exponent, not correctly rounded.
// The integer part is accumulated as number*10 + digit and each fraction digit is added
// as digit*scale with scale *= 0.1f.  The reference is compiled with -ffast-math, under
// which GCC folds (number*10 + c) - '0' into number*10 + (c - '0'); the fixtures built
// from the reference pin this form.
float Stof(const char* s, size_t n) {
    float number = 0.0f;
    bool neg = false, dot = false;
    float scale = 0.1f;
    for (size_t j = 0; j < n; j++) {
        char c = s[j];
        if (j == 0 && c == '-')
            neg = true;
        else if (!dot && c == '.')
            dot = true;
        else if (!dot)
            number = number * 10 + (float)(c - '0');
        else {
            number += (float)(c - '0') * scale;
            scale *= 0.1f;
        }
    }
    return neg ? -number : number;
}

// pstd::stoi (string.cpp:37-48): stops at '.', leading '-'.
int Stoi(const char* s, size_t n) {
    int number = 0;
    bool neg = false;
    for (size_t j = 0; j < n; j++) {
        if (s[j] == '.')
            break;
        if (j == 0 && s[j] == '-')
            neg = true;
        else
            number = number * 10 + s[j] - '0';
    }
    return neg ? -number : number;
}

// pstd::stofs / stois (string.cpp:71-120): tokens of [0-9.-]; missing components repeat
// the last value read; an empty string gives 0.
template <typename T, typename F>
static void Tokens(const std::string& str, T* ptr, int N, F&& conv, bool allowDot) {
    int dim = 0, start = -1;
    for (int i = 0; i < (int)str.size(); i++) {
        char c = str[i];
        if (IsNumber(c) || c == '-' || (allowDot && c == '.')) {
            if (start == -1)
                start = i;
        } else if (start != -1) {
            ptr[dim++] = conv(str.data() + start, (size_t)(i - start));
            start = -1;
            if (dim == N)
                return;
        }
    }
    if (start != -1)
        ptr[dim++] = conv(str.data() + start, str.size() - start);
    if (dim == 0) {
        ptr[0] = 0;
        dim++;
    }
    for (int i = dim; i < N; i++)
        ptr[i] = ptr[dim - 1];
}
void Stofs(const std::string& str, float* ptr, int N) {
    Tokens(str, ptr, N, Stof, true);
}
void Stois(const std::string& str, int* ptr, int N) {
    Tokens(str, ptr, N, Stoi, false);
}

// ---------------------------------------------------------------- Parameters
const std::string* Params::Value(const std::string& name) const {
    auto it = values.find(name);
    return it == values.end() ? nullptr : &it->second;
}
bool Params::HasValue(const std::string& name) const {
    return values.count(name) != 0;
}
bool Params::HasSubset(const std::string& name) const {
    return subset.count(name) != 0 || HasValue(name);
}
Params& Params::AddSubset(const std::string& name) {
    auto& sub = subset[name];
    sub.emplace_back();
    return sub.back();
}
// parameters.cpp:26-44: a plain value "k: v" also serves as subset k with "@" = v.
Params& Params::operator[](const std::string& name) {
    auto& ss = subset[name];
    if (HasValue(name) && ss.empty())
        AddSubset(name).values["@"] = values[name];
    if (ss.empty())
        ss.resize(1);
    return subset[name].back();
}
std::optional<std::string> Params::TryString(const std::string& name) const {
    if (auto v = Value(name))
        return *v;
    if (name == "type" && HasValue("@"))
        return values.at("@");
    return std::nullopt;
}
std::string Params::String(const std::string& name, const char* fallback) const {
    if (auto v = TryString(name))
        return *v;
    if (fallback)
        return fallback;
    throw SceneError(PG_ERR_PARSE, "[Parameters][GetString]cannot find \"" + name + "\"");
}
std::optional<float> Params::TryFloat(const std::string& name) const {
    if (auto v = Value(name))
        return Stof(v->data(), v->size());
    return std::nullopt;
}
float Params::Float(const std::string& name) const {
    if (auto v = TryFloat(name))
        return *v;
    throw SceneError(PG_ERR_PARSE, "[Parameters][GetFloat]cannot find \"" + name + "\"");
}
float Params::Float(const std::string& name, float fallback) const {
    auto v = TryFloat(name);
    return v ? *v : fallback;
}
std::optional<int> Params::TryInt(const std::string& name) const {
    if (auto v = Value(name))
        return Stoi(v->data(), v->size());
    return std::nullopt;
}
int Params::Int(const std::string& name) const {
    if (auto v = TryInt(name))
        return *v;
    throw SceneError(PG_ERR_PARSE, "[Parameters][GetInt]cannot find \"" + name + "\"");
}
int Params::Int(const std::string& name, int fallback) const {
    auto v = TryInt(name);
    return v ? *v : fallback;
}
bool Params::Bool(const std::string& name, bool fallback) const {
    auto v = Value(name);
    if (!v)
        return fallback;
    std::string s = *v;
    for (auto& c : s)
        if ('A' <= c && c <= 'Z')
            c += 'a' - 'A';
    if (s == "true")
        return true;
    if (s == "false")
        return false;
    return Stoi(s.data(), s.size()) != 0;
}
std::optional<std::array<float, 3>> Params::TryVec3(const std::string& name) const {
    auto v = Value(name);
    if (!v)
        return std::nullopt;
    std::array<float, 3> r;
    Stofs(*v, r.data(), 3);
    return r;
}
std::array<float, 3> Params::Vec3(const std::string& name) const {
    if (auto v = TryVec3(name))
        return *v;
    throw SceneError(PG_ERR_PARSE, "[Parameters][GetVec3]cannot find \"" + name + "\"");
}
std::array<float, 3> Params::Vec3(const std::string& name, std::array<float, 3> fb) const {
    auto v = TryVec3(name);
    return v ? *v : fb;
}
std::array<int, 2> Params::Vec2i(const std::string& name, std::array<int, 2> fb) const {
    auto v = Value(name);
    if (!v)
        return fb;
    std::array<int, 2> r;
    Stois(*v, r.data(), 2);
    return r;
}

std::array<float, 2> Params::Vec2(const std::string& name, std::array<float, 2> fb) const {
    auto v = Value(name);
    if (!v)
        return fb;
    std::array<float, 2> r;
    Stofs(*v, r.data(), 2);
    return r;
}

// ---------------------------------------------------------------- parser
namespace {

bool IsLetter(char s) {
    return (s >= 'A' && s <= 'z') || (s >= '0' && s <= '9') || s == '_';  // parser.cpp:17-19
}

struct View {
    const char* p;
    size_t n;
    char at(size_t i) const {
        return i < n ? p[i] : '\0';
    }
    void drop(size_t k) {
        k = std::min(k, n);
        p += k;
        n -= k;
    }
};

template <typename F>
std::optional<size_t> FirstOfF(const View& v, F&& f) {
    for (size_t i = 0; i < v.n; i++)
        if (f(v.p[i]))
            return i;
    return std::nullopt;
}

// parser.cpp:34-43: skip whitespace; a "//" comment is recognised after a whitespace
// character and runs to the end of the line.
void EscapeSpace(View& s) {
    while (s.n && IsSpace(s.p[0])) {
        s.drop(1);
        if (s.n >= 2 && s.p[0] == '/' && s.p[1] == '/') {
            while (s.n && s.p[0] != '\n' && s.p[0] != '\r')
                s.drop(1);
            s.drop(1);
        }
    }
}

Params ParseBlock(View& block, int depth) {
    if (depth > 64)
        throw SceneError(PG_ERR_PARSE, "scene nesting deeper than 64 blocks");
    Params params;
    while (true) {
        EscapeSpace(block);
        if (!FirstOfF(block, IsLetter))
            break;
        auto sep = FirstOfF(block, [](char c) { return c == ':' || c == '=' || c == '{'; });
        if (!sep)
            throw SceneError(PG_ERR_PARSE, "expected ':', '=' or '{' after a key");
        if (auto end = FirstOfF(block, [](char c) { return c == '}'; }))
            if (*sep > *end)
                break;
        auto keyEnd = FirstOfF(block, [](char c) { return !IsLetter(c); });
        if (!keyEnd)
            throw SceneError(PG_ERR_PARSE, "unterminated key");
        std::string key(block.p, *keyEnd);
        std::string name;
        for (size_t i = *keyEnd; i < *sep; i++)
            if (IsLetter(block.p[i]))
                name += block.p[i];
        block.drop(*sep);
        bool typed = false;
        std::string value;
        if (block.at(0) != '{') {
            typed = true;
            block.drop(1);
            EscapeSpace(block);
            auto valueEnd =
                FirstOfF(block, [](char c) { return c == '\n' || c == '\r' || c == '{'; });
            if (!valueEnd)
                throw SceneError(PG_ERR_PARSE, "value of \"" + key + "\" has no line end");
            value.assign(block.p, *valueEnd);
            params.values[key] = value;
            block.drop(*valueEnd);
        }
        EscapeSpace(block);
        if (block.at(0) == '{') {
            block.drop(1);
            Params sub = ParseBlock(block, depth + 1);
            Params& dst = params.AddSubset(key);
            dst = std::move(sub);
            if (typed)
                dst.values["@"] = value;
            if (!name.empty() && !dst.HasValue("name"))
                dst.values["name"] = name;
        }
    }
    if (auto end = FirstOfF(block, [](char c) { return c == '}'; }))
        block.drop(*end + 1);
    return params;
}

}  // namespace

Params ParseScene(const std::string& text) {
    View v{text.data(), text.size()};
    return ParseBlock(v, 0);
}

// ---------------------------------------------------------------- files
static std::string ReadFile(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw SceneError(PG_ERR_IO, "cannot open \"" + path + "\"");
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

// objloader.cpp:12-100 for the forms pine handles: "v x y z", "f a b c", "f a b c d" and
// the slash forms; lines are only those terminated by '\n'; indices are 1-based, negative
// ones are relative, and the smallest index is subtracted at the end.
void LoadObj(const std::string& path, std::vector<float>& verts, std::vector<uint32_t>& idx) {
    std::string raw = ReadFile(path);
    std::vector<float> v;
    std::vector<uint32_t> ind;
    size_t pos = 0;
    std::string face;
    while (true) {
        size_t nl = raw.find('\n', pos);
        if (nl == std::string::npos)
            break;
        std::string line = raw.substr(pos, nl - pos);
        pos = nl + 1;
        if (line.size() >= 2 && line[0] == 'v' && line[1] != 't' && line[1] != 'n') {
            float p[3];
            Stofs(line.substr(2), p, 3);
            v.insert(v.end(), p, p + 3);
        } else if (!line.empty() && line[0] == 'f') {
            std::string l = line.size() > 2 ? line.substr(2) : std::string();
            size_t slashes = std::count(l.begin(), l.end(), '/');
            face.clear();
            auto takeVertex = [&](bool last) {
                face += l.substr(0, l.find('/'));
                size_t sp = l.find(' ');
                l = sp == std::string::npos ? std::string() : l.substr(sp + 1);
                if (!last)
                    face += " ";
            };
            if (slashes == 0) {
                face = l;
            } else if (slashes == 6) {
                takeVertex(false), takeVertex(false), takeVertex(true);
            } else {
                takeVertex(false), takeVertex(false), takeVertex(false), takeVertex(true);
            }
            size_t spaces = std::count(face.begin(), face.end(), ' ');
            int64_t nverts = (int64_t)(v.size() / 3);
            auto fix = [&](int i) { return (uint32_t)(i < 0 ? nverts + i : i - 1); };
            if (spaces == 2) {
                int f[3];
                Stois(face, f, 3);
                ind.insert(ind.end(), {fix(f[0]), fix(f[1]), fix(f[2])});
            } else if (spaces == 3) {
                int f[4];
                Stois(face, f, 4);
                uint32_t a = fix(f[0]), b = fix(f[1]), c = fix(f[2]), d = fix(f[3]);
                ind.insert(ind.end(), {a, b, c, a, c, d});
            }
        }
    }
    if (!ind.empty()) {
        uint32_t mn = *std::min_element(ind.begin(), ind.end());
        for (auto& i : ind)
            i -= mn;
    }
    for (auto i : ind)
        if ((uint64_t)i * 3 + 2 >= v.size())
            throw SceneError(PG_ERR_PARSE, "OBJ index out of range in \"" + path + "\"");
    verts.swap(v);
    idx.swap(ind);
}

// fileio.cpp:194-202: int32 sx, sy, sz then sx*sy*sz floats, x fastest.
// Huffman-compressed 16-bit volume (the format of pine's CompressVolume /
// LoadCompressedVolume, fileio.cpp:204-249, and HuffmanEncode/HuffmanDecode,
// util/huffman.h:87-190; pine itself ships the reader commented out).  Layout:
//   int32 size[3]; uint64 treeBytes, encodedBytes;
//   tree: the raw bytes of the writer's hash map object (56 bytes; its element count at
//         byte 24), then per entry a uint16 value and its uint32 code;
//   encoded: the raw bytes of the writer's byte vector (24 bytes: begin, end, capacity
//         pointers; its length is end - begin), the bytes, uint32 bit count, uint64 count.
// A code is its bits under a leading 1 (the tree path); the stream holds each code's bits
// below that 1, least significant first, packed from bit 0 of each byte.  A voxel is its
// 16-bit value / 2047 (the writer clamped densities to 32 and scaled by 65535 / 32 in int).
void LoadCompressedVolume(const std::string& path, std::vector<float>& density, int size[3]) {
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw SceneError(PG_ERR_IO, "cannot open volume \"" + path + "\"");
    std::vector<char> all((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    auto fail = [&](const char* what) {
        throw SceneError(PG_ERR_PARSE, std::string("compressed volume \"") + path + "\": " + what);
    };
    size_t pos = 0;
    auto take = [&](void* dst, size_t n) {
        if (pos + n > all.size())
            fail("truncated");
        std::memcpy(dst, all.data() + pos, n);
        pos += n;
    };
    int32_t hdr[3];
    uint64_t treeBytes, encBytes;
    take(hdr, 12);
    take(&treeBytes, 8);
    take(&encBytes, 8);
    if (hdr[0] <= 0 || hdr[1] <= 0 || hdr[2] <= 0 || (int64_t)hdr[0] * hdr[1] * hdr[2] > (1ll << 33))
        fail("bad size");
    // Every size is checked against the bytes that remain before any arithmetic on it, so
    // no sum below can wrap around.
    const uint64_t rest = all.size() - pos;
    if (treeBytes < 56 || treeBytes > rest || (treeBytes - 56) % 6 != 0 ||
        encBytes != rest - treeBytes || encBytes < 36)
        fail("section sizes do not add up");
    const size_t treeStart = pos;
    uint64_t entries;
    std::memcpy(&entries, all.data() + treeStart + 24, 8);
    if (entries != (treeBytes - 56) / 6 || entries == 0)
        fail("code table size");
    pos = treeStart + 56;
    std::vector<uint16_t> values(entries);
    std::vector<uint32_t> codes(entries);
    for (uint64_t i = 0; i < entries; i++) {
        take(&values[i], 2);
        take(&codes[i], 4);
        if (codes[i] == 0)
            fail("empty code");
    }
    uint64_t vb[3];
    take(vb, 24);
    if (vb[1] < vb[0] || vb[1] - vb[0] != encBytes - 36)
        fail("encoded section size");
    const uint64_t nbytes = encBytes - 36;  // bounded by the file size
    const unsigned char* bits = reinterpret_cast<const unsigned char*>(all.data() + pos);
    pos += nbytes;
    uint32_t nbits;
    uint64_t count;
    take(&nbits, 4);
    take(&count, 8);
    if (count != (uint64_t)hdr[0] * hdr[1] * hdr[2] || nbits > nbytes * 8)
        fail("element or bit count");
    density.resize(count);
    if (entries == 1) {  // a single value needs no bits (huffman.h:129-134)
        std::fill(density.begin(), density.end(), values[0] / 2047.0f);
    } else {
        // Decoding trie over the codes' bits, least significant first: node 0 is the root,
        // node k's children are 2k + 1 (bit 0) and 2k + 2 (bit 1); leaf[k] = 1 + value index.
        std::vector<uint32_t> leaf(2);
        for (uint64_t i = 0; i < entries; i++) {
            uint32_t c = codes[i];
            int h = 31 - __builtin_clz(c);
            if (h == 0)
                fail("code without bits");
            size_t node = 0;
            for (int b = 0; b < h; b++) {
                node = node * 2 + ((c >> b) & 1 ? 2 : 1);
                if (node >= (size_t)1 << 26)
                    fail("code too long");
            }
            if (node >= leaf.size())
                leaf.resize(std::max(node + 1, leaf.size() * 2));
            leaf[node] = (uint32_t)i + 1;
        }
        size_t node = 0, out = 0;
        for (uint32_t b = 0; b < nbits; b++) {
            node = node * 2 + (((bits[b >> 3] >> (b & 7)) & 1) ? 2 : 1);
            if (node >= leaf.size())
                fail("bit stream leaves the code table");
            if (uint32_t v = leaf[node]) {
                if (out == count)
                    fail("more voxels than the header holds");
                density[out++] = values[v - 1] / 2047.0f;
                node = 0;
            }
        }
        if (out != count || node != 0)
            fail("bit stream ends inside the volume");
    }
    size[0] = hdr[0], size[1] = hdr[1], size[2] = hdr[2];
}

void LoadVolume(const std::string& path, std::vector<float>& density, int size[3]) {
    const std::string ext = ".compressed";
    if (path.size() > ext.size() && path.compare(path.size() - ext.size(), ext.size(), ext) == 0)
        return LoadCompressedVolume(path, density, size);
    std::ifstream f(path, std::ios::binary);
    if (!f)
        throw SceneError(PG_ERR_IO, "cannot open volume \"" + path + "\"");
    int32_t hdr[3];
    if (!f.read((char*)hdr, 12))
        throw SceneError(PG_ERR_IO, "truncated volume header in \"" + path + "\"");
    if (hdr[0] <= 0 || hdr[1] <= 0 || hdr[2] <= 0 || (int64_t)hdr[0] * hdr[1] * hdr[2] > (1ll << 33))
        throw SceneError(PG_ERR_PARSE, "bad volume size in \"" + path + "\"");
    size_t n = (size_t)hdr[0] * hdr[1] * hdr[2];
    density.resize(n);
    if (!f.read((char*)density.data(), (std::streamsize)(n * 4)))
        throw SceneError(PG_ERR_IO, "truncated volume data in \"" + path + "\"");
    size[0] = hdr[0], size[1] = hdr[1], size[2] = hdr[2];
}

// ---------------------------------------------------------------- factories
namespace {

void Warn(const std::string& msg) {
    std::fprintf(stderr, "[pine-gpu] %s\n", msg.c_str());
}

int NodeStackEffectHost(int op) {
    return NodeStackEffect(op);
}

// node.cpp:33-97 for a constant node: "k: v" literal values and Constant{float vec3}.
struct ConstNode {
    float f;
    std::array<float, 3> v;
};
ConstNode CreateNode(Params& p, const std::string& what) {
    std::string type = p.String("type", "");
    if (type == "Constant")
        return {p.Float("float"), p.Vec3("vec3")};
    static const char* kTextured[] = {"Position", "Normal",   "TexCoord",     "Decompose",
                                      "Composite", "Add",     "Substract",    "Multiply",
                                      "Divide",    "MultiplyAdd", "Length",   "Sqr",
                                      "Sqrt",      "Pow",     "Sin",          "Cos",
                                      "Tan",       "Fract",   "Checkerboard", "Noise",
                                      "Noise3D",   "Texture", "Invert"};
    for (auto t : kTextured)
        if (type == t)
            throw SceneError(PG_ERR_UNSUPPORTED,
                             "texture node \"" + type + "\" (" + what + ") is not supported");
    if (p.HasValue("@") && !p.values["@"].empty()) {
        // The literal case (node.cpp:89-91): float from stof of the whole text, vec3 from
        // stofs.  Only EvalVec3 of albedo/color and EvalFloat of scalars are ever used.
        ConstNode n;
        n.f = p.Float("float", p.Float("@"));
        n.v = p.Vec3("vec3", p.Vec3("@"));
        return n;
    }
    if (type.empty())
        throw SceneError(PG_ERR_PARSE, "[Parameters][GetString]cannot find \"type\" (" + what + ")");
    Warn("[NodeInput][Create]Unknown type \"" + type + "\"");
    return {p.Float("float", 0.5f), p.Vec3("vec3", {0.5f, 0.5f, 0.5f})};
}

// node.cpp:33-97 in full: the node graph at p, compiled into a postfix program for pine's
// EvalVec3 (vec) or EvalFloat.  The two differ for some nodes: Position, Normal, TexCoord
// and Composite have no float value (0, Node::EvalFloat), Constant yields its float or its
// vec3, Noise3D is Turbulence as a float and Turbulence3D as a vec3; inputs that pine reads
// with EvalFloat (frequency, octaves, exponents, Composite's parts) are compiled as floats.
void EmitNode(Params& p, bool vec, std::vector<pg_node_op>& ops, const std::string& what, int depth) {
    if (depth > 64)
        throw SceneError(PG_ERR_UNSUPPORTED, "node graph of " + what + " nested too deeply");
    auto op = [&](int code, int arg = 0) {
        pg_node_op o{};
        o.op = code;
        o.arg = arg;
        ops.push_back(o);
    };
    auto constant = [&](float f, std::array<float, 3> v) {
        pg_node_op o{};
        o.op = PG_NODE_CONST;
        if (vec)
            o.c[0] = v[0], o.c[1] = v[1], o.c[2] = v[2];
        else
            o.c[0] = o.c[1] = o.c[2] = f;
        ops.push_back(o);
    };
    auto zero = [&]() { constant(0.0f, {0.0f, 0.0f, 0.0f}); };
    auto emit = [&](const char* input, bool v) { EmitNode(p[input], v, ops, what, depth + 1); };
    const std::string type = p.String("type", "");
    struct Unary {
        const char* name;
        int code;
    };
    static const Unary kUnary[] = {{"Sqr", PG_NODE_SQR},   {"Sqrt", PG_NODE_SQRT},   {"Sin", PG_NODE_SIN},
                                   {"Cos", PG_NODE_COS},   {"Tan", PG_NODE_TAN},     {"Fract", PG_NODE_FRACT},
                                   {"Invert", PG_NODE_INVERT}};
    static const Unary kBinary[] = {{"Add", PG_NODE_ADD},
                                    {"Substract", PG_NODE_SUB},
                                    {"Multiply", PG_NODE_MUL},
                                    {"Divide", PG_NODE_DIV}};
    if (type == "Constant")
        return constant(p.Float("float"), p.Vec3("vec3"));
    if (type == "Position")
        return vec ? op(PG_NODE_POSITION) : zero();
    if (type == "Normal")
        return vec ? op(PG_NODE_NORMAL) : zero();
    if (type == "TexCoord")
        return vec ? op(PG_NODE_TEXCOORD) : zero();
    if (type == "Decompose") {
        int dim = p.Int("dimension");
        if (dim < 0 || dim > 2)
            throw SceneError(PG_ERR_PARSE, "Decompose dimension out of range (" + what + ")");
        emit("input", true);
        return op(PG_NODE_DECOMPOSE, dim);
    }
    if (type == "Composite") {
        if (!vec)
            return zero();
        emit("inputX", false);
        emit("inputY", false);
        emit("inputZ", false);
        return op(PG_NODE_COMPOSITE);
    }
    for (const Unary& b : kBinary)
        if (type == b.name) {
            emit("input", vec);
            emit("factor", vec);
            return op(b.code);
        }
    if (type == "MultiplyAdd") {
        emit("input", vec);
        emit("mulFactor", vec);
        emit("addFactor", vec);
        return op(PG_NODE_MULADD);
    }
    if (type == "Length") {
        emit("input", true);
        return op(PG_NODE_LENGTH);
    }
    for (const Unary& u : kUnary)
        if (type == u.name) {
            emit("input", vec);
            return op(u.code);
        }
    if (type == "Pow") {
        emit("input", vec);
        emit("exp", false);
        return op(PG_NODE_POW);
    }
    if (type == "Checkerboard") {
        emit("input", true);
        emit("frequency", false);
        return op(PG_NODE_CHECKER);
    }
    if (type == "Noise" || type == "Noise3D") {
        emit("input", true);
        emit("frequency", false);
        emit("octaves", false);
        return op(type == "Noise3D" && vec ? PG_NODE_NOISE3D : PG_NODE_NOISE);
    }
    if (type == "Texture")
        throw SceneError(PG_ERR_UNSUPPORTED, "Texture nodes (image files) are not supported (" + what + ")");
    if (p.HasValue("@") && !p.values["@"].empty())
        // The literal case (node.cpp:89-91): float from stof of the whole text, vec3 from stofs.
        return constant(p.Float("float", p.Float("@")), p.Vec3("vec3", p.Vec3("@")));
    if (type.empty())
        throw SceneError(PG_ERR_PARSE, "[Parameters][GetString]cannot find \"type\" (" + what + ")");
    Warn("[NodeInput][Create]Unknown type \"" + type + "\"");
    return constant(p.Float("float", 0.5f), p.Vec3("vec3", {0.5f, 0.5f, 0.5f}));
}

// A BSDF or material parameter: the constant node's value (returns 0), or 1 + the first op
// of its program in s.node_ops.
int NodeParam(Params& p, bool vec, HostScene& s, const std::string& what, float& f,
              std::array<float, 3>& v) {
    std::vector<pg_node_op> prog;
    EmitNode(p, vec, prog, what, 0);
    if (prog.size() == 1 && prog[0].op == PG_NODE_CONST) {
        f = prog[0].c[0];
        v = {prog[0].c[0], prog[0].c[1], prog[0].c[2]};
        return 0;
    }
    int depth = 0, maxDepth = 0;
    for (const pg_node_op& o : prog) {
        depth += NodeStackEffectHost(o.op);
        maxDepth = std::max(maxDepth, depth);
    }
    if ((int)prog.size() + 1 > PG_NODE_MAX_OPS || maxDepth > PG_NODE_MAX_STACK)
        throw SceneError(PG_ERR_UNSUPPORTED, "node graph of " + what + " is too large");
    pg_node_op end{};
    end.op = PG_NODE_END;
    prog.push_back(end);
    int start = (int)s.node_ops.size();
    s.node_ops.insert(s.node_ops.end(), prog.begin(), prog.end());
    return start + 1;
}

pg_bsdf CreateBSDF(Params& p, HostScene& s) {
    std::string type = p.String("type");
    pg_bsdf b{};
    if (type == "Conductor") {
        b.type = PG_BSDF_CONDUCTOR;
    } else if (type == "Dielectric") {
        b.type = PG_BSDF_DIELECTRIC;
    } else {
        if (type != "Diffuse")
            Warn("[BSDF][Create]Unknown type \"" + type + "\"");
        b.type = PG_BSDF_DIFFUSE;
    }
    float f;
    std::array<float, 3> v;
    if (b.type == PG_BSDF_DIELECTRIC && !p.HasSubset("albedo")) {
        b.albedo[0] = b.albedo[1] = b.albedo[2] = 1.0f;  // bxdf.cpp:176-181
    } else {
        b.albedo_node = NodeParam(p["albedo"], true, s, "albedo", f, v);
        std::copy(v.begin(), v.end(), b.albedo);
    }
    if (b.type != PG_BSDF_DIFFUSE) {
        b.roughness_node = NodeParam(p["roughness"], false, s, "roughness", f, v);
        b.roughness = f;
    }
    if (b.type == PG_BSDF_DIELECTRIC) {
        b.eta_node = NodeParam(p["eta"], false, s, "eta", f, v);
        b.eta = f;
    }
    return b;
}

pg_material CreateMaterial(Params& p, HostScene& s) {
    std::string type = p.String("type");
    pg_material m{};
    if (p.HasSubset("bumpMap")) {
        // Every bump map is a program, a constant one included: BumpNormal rebuilds the
        // normal from dpdu x dpdv even when the map is flat (material.cpp:46-60).
        std::vector<pg_node_op> prog;
        EmitNode(p["bumpMap"], false, prog, "bumpMap", 0);
        int depth = 0, maxDepth = 0;
        for (const pg_node_op& o : prog) {
            depth += NodeStackEffectHost(o.op);
            maxDepth = std::max(maxDepth, depth);
        }
        if ((int)prog.size() + 1 > PG_NODE_MAX_OPS || maxDepth > PG_NODE_MAX_STACK)
            throw SceneError(PG_ERR_UNSUPPORTED, "bump map node graph is too large");
        pg_node_op end{};
        prog.push_back(end);
        m.bump_node = (int)s.node_ops.size() + 1;
        s.node_ops.insert(s.node_ops.end(), prog.begin(), prog.end());
    }
    if (type == "Emissive") {
        m.type = PG_MATERIAL_EMISSIVE;
        ConstNode c = CreateNode(p["color"], "color");
        std::copy(c.v.begin(), c.v.end(), m.emission);
        return m;
    }
    if (type != "Layered")
        Warn("[Material][Create]Unknown type \"" + type + "\"");
    m.type = PG_MATERIAL_LAYERED;
    // material.cpp:33-43: "layerN" subsets, ordered by N descending (top layer first).
    std::vector<std::pair<int, Params*>> layers;
    for (auto& kv : p.subset)
        if (kv.first.compare(0, 5, "layer") == 0 && !kv.second.empty())
            layers.push_back({Stoi(kv.first.data() + 5, kv.first.size() - 5), &kv.second.back()});
    std::stable_sort(layers.begin(), layers.end(),
                     [](const auto& a, const auto& b) { return a.first > b.first; });
    if ((int)layers.size() > PG_MAX_LAYERS)
        throw SceneError(PG_ERR_UNSUPPORTED, "more than 4 layers in a material");
    for (auto& l : layers)
        m.layers[m.num_layers++] = CreateBSDF(*l.second, s);
    return m;
}

}  // namespace

void LoadSceneFile(const std::string& path, HostScene& s) {
    std::string text = ReadFile(path);
    Params params = ParseScene(text);
    // fileio.cpp:40-48,256: every file in the scene is relative to the scene's directory.
    std::string dir;
    size_t slash = path.find_last_of('/');
    dir = slash == std::string::npos ? std::string("./") : path.substr(0, slash + 1);

    std::map<std::string, int> materials, media;
    for (auto& p : params.subset["Material"]) {
        materials[p.String("name")] = (int)s.materials.size();
        s.materials.push_back(CreateMaterial(p, s));
    }
    for (auto& p : params.subset["Medium"]) {
        std::string type = p.String("type");
        pg_medium m{};
        m.g = p.Float("g", 0.0f);
        auto sa = p.Vec3("sigma_a"), ss = p.Vec3("sigma_s");
        std::copy(sa.begin(), sa.end(), m.sigma_a);
        std::copy(ss.begin(), ss.end(), m.sigma_s);
        if (type == "Grid") {
            m.type = PG_MEDIUM_GRID;
            s.densities.emplace_back();
            LoadVolume(dir + p.String("file"), s.densities.back(), m.size);
            auto pos = p.Vec3("position");
            std::copy(pos.begin(), pos.end(), m.position);
            m.scale = p.Float("scale", 1.0f);
            m.interpolate = p.Bool("interpolate", true) ? 1 : 0;
            std::string method = p.String("samplingMethod", "deltaTracking");
            if (method != "deltaTracking")
                throw SceneError(PG_ERR_UNSUPPORTED, "grid sampling method \"" + method + "\"");
        } else {
            if (type != "Homogeneous")
                Warn("[Medium][Create]Unknown type \"" + type + "\"");
            m.type = PG_MEDIUM_HOMOGENEOUS;
            s.densities.emplace_back();
        }
        media[p.String("name")] = (int)s.media.size();
        s.media.push_back(m);
    }
    for (auto& p : params.subset["Light"]) {
        std::string type = p.String("type");
        pg_light l{};
        if (type == "Directional") {
            l.type = PG_LIGHT_DIRECTIONAL;
            auto d = p.Vec3("direction"), c = p.Vec3("color");
            std::copy(d.begin(), d.end(), l.p);
            std::copy(c.begin(), c.end(), l.p + 3);
        } else if (type == "Environment") {
            Params& e = p["environment"];
            std::string et = e.String("type");
            if (et == "Sky") {
                l.type = PG_LIGHT_SKY;
                auto d = e.Vec3("sunDirection"), c = e.Vec3("sunColor");
                std::copy(d.begin(), d.end(), l.p);
                std::copy(c.begin(), c.end(), l.p + 3);
            } else if (et == "Constant") {
                l.type = PG_LIGHT_CONSTANT_ENV;
                auto c = e.Vec3("color");
                std::copy(c.begin(), c.end(), l.p + 3);
            } else {
                throw SceneError(PG_ERR_UNSUPPORTED, "environment \"" + et + "\" is not supported");
            }
        } else {
            if (type != "Point")
                Warn("[Light][Create]Unknown type \"" + type + "\"");
            l.type = PG_LIGHT_POINT;
            auto q = p.Vec3("position"), c = p.Vec3("color");
            std::copy(q.begin(), q.end(), l.p);
            std::copy(c.begin(), c.end(), l.p + 3);
        }
        s.lights.push_back(l);
    }
    for (auto& p : params.subset["Shape"]) {
        std::string type = p.String("type");
        pg_shape sh{};
        sh.material = -1;
        sh.medium_inside = sh.medium_outside = -1;
        auto put = [&](int off, std::array<float, 3> v) {
            std::copy(v.begin(), v.end(), sh.p + off);
        };
        if (type == "Plane") {
            sh.type = PG_SHAPE_PLANE;
            put(0, p.Vec3("position"));
            // Plane::Create normalises with pine's sqrt (geometry.cpp:346-348).
            auto n = p.Vec3("normal");
            V3 nn = Normalize<kPine>(v3(n[0], n[1], n[2]));
            put(3, {nn.x, nn.y, nn.z});
        } else if (type == "Triangle") {
            sh.type = PG_SHAPE_TRIANGLE;
            put(0, p.Vec3("v0")), put(3, p.Vec3("v1")), put(6, p.Vec3("v2"));
        } else if (type == "Rect") {
            sh.type = PG_SHAPE_RECT;
            put(0, p.Vec3("position")), put(3, p.Vec3("ex")), put(6, p.Vec3("ey"));
        } else if (type == "TriangleMesh") {
            sh.type = PG_SHAPE_MESH;
            std::vector<float> v;
            std::vector<uint32_t> ind;
            LoadObj(dir + p.String("file"), v, ind);
            if (auto sc = p.TryVec3("scale"))
                for (size_t i = 0; i < v.size(); i++)
                    v[i] *= (*sc)[i % 3];
            if (auto ps = p.TryVec3("position"))
                for (size_t i = 0; i < v.size(); i++)
                    v[i] += (*ps)[i % 3];
            uint32_t base = (uint32_t)(s.vertices.size() / 3);
            sh.mesh_first_triangle = (int64_t)(s.indices.size() / 3);
            sh.mesh_num_triangles = (int64_t)(ind.size() / 3);
            s.vertices.insert(s.vertices.end(), v.begin(), v.end());
            for (auto i : ind)
                s.indices.push_back(i + base);
        } else if (type == "Cylinder" || type == "Disk" || type == "Line") {
            throw SceneError(PG_ERR_UNSUPPORTED, "shape \"" + type + "\" is not supported");
        } else {
            if (type != "Sphere")
                Warn("[Shape][Create]Unknown type \"" + type + "\"");
            sh.type = PG_SHAPE_SPHERE;
            put(0, p.Vec3("position"));
            sh.p[3] = p.Float("radius");
        }
        if (auto name = p.TryString("material")) {
            auto it = materials.find(*name);
            if (it == materials.end())
                throw SceneError(PG_ERR_PARSE, "[Shape][Create]Material \"" + *name + "\" is not found");
            sh.material = it->second;
        }
        auto medium = [&](const char* key, int& slot) {
            if (auto name = p.TryString(key)) {
                auto it = media.find(*name);
                if (it == media.end())
                    throw SceneError(PG_ERR_PARSE, "[Shape][Create]Medium \"" + *name + "\" is not found");
                slot = it->second;
            }
        };
        medium("medium", sh.medium_inside);
        medium("mediumInside", sh.medium_inside);
        medium("mediumOutside", sh.medium_outside);
        s.shapes.push_back(sh);
    }

    // Camera (camera.cpp:86-107) and film (film.cpp:7-12).
    Params& cam = params["Camera"];
    std::string ctype = cam.String("type", "ThinLen");
    if (ctype != "ThinLen")
        Warn("[Camera][Create]Unknown type \"" + ctype + "\"");
    Params& film = cam["film"];
    auto size = film.Vec2i("size", {720, 480});
    pg_camera& c = s.camera;
    auto from = cam.Vec3("from"), to = cam.Vec3("to");
    std::copy(from.begin(), from.end(), c.from);
    std::copy(to.begin(), to.end(), c.to);
    c.fov = cam.Float("fov");
    c.lens_radius = cam.Float("lensRadius", 0.0f);
    c.focus_distance = cam.Float("focusDistance", 1.0f);
    c.width = size[0];
    c.height = size[1];
    c.medium = -1;
    if (auto name = cam.TryString("medium")) {
        auto it = media.find(*name);
        if (it == media.end())
            throw SceneError(PG_ERR_PARSE, "[Camera][Create]Medium \"" + *name + "\" is not found");
        c.medium = it->second;
    }
    if (c.width <= 0 || c.height <= 0)
        throw SceneError(PG_ERR_PARSE, "film size must be positive");

    // Integrator (integrator.cpp:20-56): maxDepth default 4, sampler spp, light sampler.
    Params& integ = params["Integrator"];
    std::string itype = integ.String("type", "Path");
    s.integrator = itype == "RandomWalk" ? PG_INTEGRATOR_RANDOM_WALK : PG_INTEGRATOR_PATH;
    if (itype != "Path" && itype != "GpuPath" && itype != "RandomWalk")
        Warn("[Integrator][Create]Integrator \"" + itype + "\" is rendered as GpuPath");
    s.max_depth = integ.Int("maxDepth", 4);
    // Sampler (CreateSampler, sampler.cpp:281-293) and its samples per pixel.
    Params& smp = integ["sampler"];
    std::string stype = smp.String("type", "Uniform");
    s.sampler = PG_SAMPLER_INDEPENDENT;
    if (stype == "Stratified") {
        s.spp = smp.Int("xPixelSamples", 1) * smp.Int("yPixelSamples", 1);
    } else if (stype == "ZeroTwoSequence") {
        int n = smp.Int("samplesPerPixel", 1), r = 1;
        while (r < n)
            r <<= 1;  // pstd::roundup2 (sampler.cpp:98-99)
        s.spp = r;
    } else {
        if (stype == "Halton") {
            s.sampler = PG_SAMPLER_HALTON;
            // randomizeStrategy: "none" or "permutateDigits"; anything else keeps the
            // default (sampler.cpp:252-259).
            s.sampler_scramble = smp.String("randomizeStrategy", "permutateDigits") != "none";
        } else if (stype == "Sobol") {
            s.sampler = PG_SAMPLER_SOBOL;
            // SobolSampler::Create (sampler.cpp:268-277): BinaryPermutate unless the string
            // names another strategy; the string's default is "fastOwen".
            std::string rs = smp.String("randomizeStrategy", "fastOwen");
            s.sampler_scramble = rs == "none"       ? PG_SOBOL_NONE
                                 : rs == "fastOwen" ? PG_SOBOL_FAST_OWEN
                                 : rs == "Owen"     ? PG_SOBOL_OWEN
                                                    : PG_SOBOL_BINARY_PERMUTATE;
        } else if (stype != "Uniform") {
            Warn("[Sampler][Create]Unknown type \"" + stype + "\"");
        }
        s.spp = smp.Int("samplesPerPixel", 1);
    }
    // Film filter (CreateFilter, filter.cpp:5-21): LanczosSinc of radius 0.5 by default.
    Params& flt = film["filter"];
    std::string ftype = flt.String("type", "LanczosSinc");
    auto radius = flt.Vec2("radius", {0.5f, 0.5f});
    s.filter_radius[0] = radius[0];
    s.filter_radius[1] = radius[1];
    s.filter_params[0] = s.filter_params[1] = 0.0f;
    if (ftype == "Box") {
        s.filter = PG_FILTER_BOX;
    } else if (ftype == "Triangle") {
        s.filter = PG_FILTER_TRIANGLE;
    } else if (ftype == "Gaussian") {
        s.filter = PG_FILTER_GAUSSIAN;
        s.filter_params[0] = flt.Float("alpha", 1.0f);
    } else if (ftype == "Mitchell") {
        s.filter = PG_FILTER_MITCHELL;
        s.filter_params[0] = flt.Float("B", 1 / 3.0f);
        s.filter_params[1] = flt.Float("C", 1.0f / 3.0f);
    } else if (ftype == "LanczosSinc") {
        s.filter = PG_FILTER_LANCZOS_SINC;
        s.filter_params[0] = flt.Float("tau", 3.0f);
    } else {
        Warn("[Filter][Create]Unknown type \"" + ftype + "\"");
        s.filter = PG_FILTER_BOX;
    }
    std::string ls = integ["lightSampler"].String("type", "Power");
    s.light_sampler = ls == "Uniform" ? PG_LIGHT_SAMPLER_UNIFORM : PG_LIGHT_SAMPLER_POWER;
}

void HostScene::Describe(pg_scene_desc& d) {
    std::memset(&d, 0, sizeof(d));
    for (size_t i = 0; i < media.size(); i++)
        media[i].density = densities[i].empty() ? nullptr : densities[i].data();
    d.num_shapes = (int32_t)shapes.size();
    d.shapes = shapes.data();
    d.num_vertices = (int64_t)(vertices.size() / 3);
    d.vertices = vertices.data();
    d.num_triangles = (int64_t)(indices.size() / 3);
    d.indices = indices.data();
    d.num_materials = (int32_t)materials.size();
    d.materials = materials.data();
    d.num_media = (int32_t)media.size();
    d.media = media.data();
    d.num_lights = (int32_t)lights.size();
    d.lights = lights.data();
    d.camera = camera;
    d.light_sampler = light_sampler;
    d.max_depth = max_depth;
    d.samples_per_pixel = spp;
    d.num_node_ops = (int32_t)node_ops.size();
    d.node_ops = node_ops.data();
    d.sampler = sampler;
    d.sampler_scramble = sampler_scramble;
    d.filter = filter;
    d.integrator = integrator;
    for (int k = 0; k < 2; k++) {
        d.filter_radius[k] = filter_radius[k];
        d.filter_params[k] = filter_params[k];
    }
}

}  // namespace pg

extern "C" float pg_pstd_stof(const char* str, int64_t len) {
    if (!str || len < 0)
        return 0.0f;
    return pg::Stof(str, (size_t)len);
}
