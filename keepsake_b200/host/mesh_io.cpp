// Mesh files of the small_pt task's mesh assets: Wavefront OBJ and keepsake's binary mesh asset.
#include "mesh_io.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <tuple>

namespace fs = std::filesystem;

namespace ksb
{
namespace mesh
{

namespace
{

constexpr const char kBinaryMagic[] = "i_am_a_binary_mesh_asset";
constexpr size_t kMagicLen = sizeof(kBinaryMagic) - 1;

// OBJ index: 1-based, or negative = relative to the end of the list so far; 0 = absent.
long obj_index(const std::string &tok, long count, const std::string &where)
{
    if (tok.empty())
        return -1;
    char *end = nullptr;
    const long i = std::strtol(tok.c_str(), &end, 10);
    if (end == tok.c_str() || *end != 0 || i == 0)
        throw Error(where + ": bad face index '" + tok + "'");
    const long v = i < 0 ? count + i : i - 1;
    if (v < 0 || v >= count)
        throw Error(where + ": face index out of range");
    return v;
}

} // namespace

std::vector<MeshData> load_obj(const fs::path &path, bool twosided, bool use_smooth_normal)
{
    std::ifstream f(path);
    if (!f)
        throw Error("cannot open " + path.string());
    std::vector<float> pos, tex, nrm;
    std::vector<MeshData> out;
    MeshData cur;
    std::map<std::tuple<long, long, long>, uint32_t> remap;
    int has_tc = -1, has_n = -1; // per mesh: -1 undecided, 0 none, 1 all
    std::string name;
    auto flush = [&]() {
        if (!cur.indices.empty()) {
            cur.twosided = twosided;
            cur.use_smooth_normal = use_smooth_normal;
            cur.name = name;
            out.push_back(std::move(cur));
        }
        cur = MeshData();
        remap.clear();
        has_tc = has_n = -1;
    };
    std::string line;
    int ln = 0;
    while (std::getline(f, line)) {
        ++ln;
        const std::string where = path.string() + ":" + std::to_string(ln);
        std::istringstream ss(line);
        std::string tag;
        ss >> tag;
        if (tag == "v" || tag == "vn") {
            float x, y, z;
            if (!(ss >> x >> y >> z))
                throw Error(where + ": bad " + tag);
            (tag == "v" ? pos : nrm).insert((tag == "v" ? pos : nrm).end(), {x, y, z});
        } else if (tag == "vt") {
            float u, v = 0.0f;
            if (!(ss >> u))
                throw Error(where + ": bad vt");
            ss >> v;
            tex.insert(tex.end(), {u, v});
        } else if (tag == "o" || tag == "g") {
            flush();
            std::getline(ss >> std::ws, name);
        } else if (tag == "f") {
            std::vector<uint32_t> poly;
            std::string tok;
            while (ss >> tok) {
                std::string parts[3];
                size_t k = 0, start = 0;
                for (size_t i = 0; i <= tok.size() && k < 3; ++i)
                    if (i == tok.size() || tok[i] == '/') {
                        parts[k++] = tok.substr(start, i - start);
                        start = i + 1;
                    }
                const long vi = obj_index(parts[0], (long)pos.size() / 3, where);
                if (vi < 0)
                    throw Error(where + ": face corner without a position");
                const long ti = obj_index(parts[1], (long)tex.size() / 2, where);
                const long ni = obj_index(parts[2], (long)nrm.size() / 3, where);
                const int tc = ti >= 0, nn = ni >= 0;
                if ((has_tc >= 0 && has_tc != tc) || (has_n >= 0 && has_n != nn))
                    throw Error(where + ": either all or no corners of a mesh have texcoords (normals)");
                has_tc = tc;
                has_n = nn;
                auto ins = remap.emplace(std::make_tuple(vi, ti, ni), cur.vertex_count());
                if (ins.second) {
                    cur.vertices.insert(cur.vertices.end(), {pos[3 * vi], pos[3 * vi + 1], pos[3 * vi + 2]});
                    if (tc)
                        cur.texcoords.insert(cur.texcoords.end(), {tex[2 * ti], tex[2 * ti + 1]});
                    if (nn)
                        cur.normals.insert(cur.normals.end(), {nrm[3 * ni], nrm[3 * ni + 1], nrm[3 * ni + 2]});
                }
                poly.push_back(ins.first->second);
            }
            if (poly.size() < 3)
                throw Error(where + ": face with fewer than 3 corners");
            for (size_t k = 2; k < poly.size(); ++k)
                cur.indices.insert(cur.indices.end(), {poly[0], poly[k - 1], poly[k]});
        }
    }
    flush();
    if (out.empty())
        throw Error(path.string() + ": no faces");
    return out;
}

namespace
{

struct Reader
{
    std::ifstream f;
    std::string where;
    template <class T>
    T get()
    {
        T v;
        f.read(reinterpret_cast<char *>(&v), sizeof(T));
        if (!f)
            throw Error(where + ": truncated binary mesh asset");
        return v;
    }
    template <class T>
    void array(std::vector<T> &v, size_t n)
    {
        v.resize(n);
        f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(sizeof(T) * n));
        if (!f)
            throw Error(where + ": truncated binary mesh asset");
    }
};

} // namespace

std::vector<MeshData> load_binary(const fs::path &path)
{
    Reader r{std::ifstream(path, std::ios::binary), path.string()};
    if (!r.f)
        throw Error("cannot open " + path.string());
    char magic[kMagicLen];
    r.f.read(magic, kMagicLen);
    if (!r.f || std::memcmp(magic, kBinaryMagic, kMagicLen) != 0)
        throw Error(path.string() + ": invalid binary mesh asset");
    const int32_t n = r.get<int32_t>();
    if (n < 0)
        throw Error(path.string() + ": invalid binary mesh asset");
    std::vector<MeshData> out((size_t)n);
    for (MeshData &m : out) {
        m.twosided = r.get<uint8_t>() != 0;
        m.use_smooth_normal = r.get<uint8_t>() != 0;
        const int32_t nv = r.get<int32_t>(), nt = r.get<int32_t>();
        const bool tc = r.get<uint8_t>() != 0, vn = r.get<uint8_t>() != 0;
        if (nv < 0 || nt < 0)
            throw Error(path.string() + ": invalid binary mesh asset");
        r.array(m.vertices, 3 * (size_t)nv + 1);
        m.vertices.pop_back(); // padding
        r.array(m.indices, 3 * (size_t)nt);
        for (uint32_t i : m.indices)
            if (i >= (uint32_t)nv)
                throw Error(path.string() + ": vertex index out of range");
        if (tc) {
            r.array(m.texcoords, 2 * (size_t)nv + 2);
            m.texcoords.resize(2 * (size_t)nv);
        }
        if (vn) {
            r.array(m.normals, 3 * (size_t)nv + 1);
            m.normals.pop_back();
        }
    }
    return out;
}

void write_binary(const fs::path &path, const std::vector<MeshData> &meshes)
{
    std::ofstream f(path, std::ios::binary);
    if (!f)
        throw Error("cannot write " + path.string());
    auto put = [&](const void *p, size_t n) { f.write(reinterpret_cast<const char *>(p), (std::streamsize)n); };
    const float nan = std::nanf("");
    put(kBinaryMagic, kMagicLen);
    const int32_t n = (int32_t)meshes.size();
    put(&n, 4);
    for (const MeshData &m : meshes) {
        const uint8_t flags[2] = {(uint8_t)m.twosided, (uint8_t)m.use_smooth_normal};
        put(flags, 2);
        const int32_t nv = (int32_t)m.vertex_count(), nt = (int32_t)m.tri_count();
        put(&nv, 4);
        put(&nt, 4);
        const uint8_t has[2] = {(uint8_t)!m.texcoords.empty(), (uint8_t)!m.normals.empty()};
        put(has, 2);
        // the arrays with the reference's padding floats (NaN, as its OBJ loader appends them)
        put(m.vertices.data(), sizeof(float) * m.vertices.size());
        put(&nan, 4);
        put(m.indices.data(), sizeof(uint32_t) * m.indices.size());
        if (has[0]) {
            put(m.texcoords.data(), sizeof(float) * m.texcoords.size());
            put(&nan, 4);
            put(&nan, 4);
        }
        if (has[1]) {
            put(m.normals.data(), sizeof(float) * m.normals.size());
            put(&nan, 4);
        }
    }
    if (!f)
        throw Error("cannot write " + path.string());
}

void transform(std::vector<MeshData> &meshes, const float m[16])
{
    // inverse transpose of the 3x3 block (cofactors / determinant)
    double a[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            a[r][c] = m[4 * r + c];
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                       a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                       a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    if (!(std::fabs(det) > 0.0))
        throw Error("to_world: singular transform");
    float it[3][3]; // (A^-1)^T = cofactor(A) / det
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
            it[r][c] = (float)((a[r1][c1] * a[r2][c2] - a[r1][c2] * a[r2][c1]) / det);
        }
    for (MeshData &md : meshes) {
        for (size_t i = 0; i + 2 < md.vertices.size(); i += 3) {
            const float x = md.vertices[i], y = md.vertices[i + 1], z = md.vertices[i + 2];
            for (int r = 0; r < 3; ++r)
                md.vertices[i + r] = m[4 * r] * x + m[4 * r + 1] * y + m[4 * r + 2] * z + m[4 * r + 3];
        }
        for (size_t i = 0; i + 2 < md.normals.size(); i += 3) {
            const float x = md.normals[i], y = md.normals[i + 1], z = md.normals[i + 2];
            float n[3];
            for (int r = 0; r < 3; ++r)
                n[r] = it[r][0] * x + it[r][1] * y + it[r][2] * z;
            const float len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            for (int r = 0; r < 3; ++r)
                md.normals[i + r] = n[r] / len;
        }
    }
}

} // namespace mesh
} // namespace ksb
