// Scene host: config reader, OBJ loader, Audio / Manual objects, object collection.
#include "scene.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>

namespace pppm_host
{

// ------------------------------------------------------------------ config --------------
namespace
{
std::string trim_blank_quote(const std::string &s)
{
    auto skip = [](char ch) { return std::isblank((unsigned char)ch) || ch == '"' || ch == '\r'; };
    size_t b = 0, e = s.size();
    while (b < e && skip(s[b]))
        b++;
    while (e > b && skip(s[e - 1]))
        e--;
    return s.substr(b, e - b);
}

// "key: value," -> key, value (simple_json_reader.h:66-72: the first ':' splits, a ',' ends
// the value, blanks and quotes trimmed)
void key_value(const std::string &line, std::string &key, std::string &value)
{
    size_t d1 = line.find(':');
    size_t d2 = std::min(line.find(','), line.size());
    if (d1 == std::string::npos)
    {
        key = trim_blank_quote(line);
        value.clear();
        return;
    }
    key = trim_blank_quote(line.substr(0, d1));
    value = d2 > d1 ? trim_blank_quote(line.substr(d1 + 1, d2 - d1 - 1)) : std::string();
}
}  // namespace

bool SceneConfig::load(const std::string &path, std::string &err)
{
    std::ifstream in(path);
    if (!in.good())
    {
        err = "cannot open config " + path;
        return false;
    }
    std::string line, key, value;
    if (!std::getline(in, line) || trim_blank_quote(line) != "{")
    {
        err = "config must start with a '{' line";
        return false;
    }
    for (int i = 0; i < 2; i++)
    {
        if (!std::getline(in, line))
        {
            err = "config ends before the two directory lines";
            return false;
        }
        key_value(line, key, value);
        dirs[key] = value;
    }
    while (true)
    {
        if (!std::getline(in, line))
        {
            err = "config ends before the object list '['";
            return false;
        }
        if (line.find('[') != std::string::npos)
            break;
        key_value(line, key, value);
        if (key.empty())
            continue;
        try
        {
            nums[key] = std::stof(value);
        }
        catch (...)
        {
            err = "numeric value expected for key " + key;
            return false;
        }
    }
    while (true)
    {
        if (!std::getline(in, line))
        {
            err = "config ends before the closing ']'";
            return false;
        }
        if (line.find(']') != std::string::npos)
            break;
        std::map<std::string, std::string> obj;
        for (int i = 0; i < 2; i++)
        {
            if (!std::getline(in, line))
            {
                err = "truncated object entry";
                return false;
            }
            key_value(line, key, value);
            obj[key] = value;
        }
        std::getline(in, line);  // the object's closing brace line
        objects.push_back(obj);
    }
    return true;
}

float SceneConfig::num(const std::string &key) const
{
    auto it = nums.find(key);
    return it == nums.end() ? 0.0f : it->second;
}

// ------------------------------------------------------------------ OBJ ------------------
bool Mesh::load_obj(const std::string &path, std::string &err)
{
    std::ifstream in(path);
    if (!in.good())
    {
        err = "cannot open mesh " + path;
        return false;
    }
    std::string line;
    while (std::getline(in, line))
    {
        std::istringstream ss(line);
        std::string tag;
        if (!(ss >> tag))
            continue;
        if (tag == "v")
        {
            Vec3 p{0, 0, 0};
            ss >> p[0] >> p[1] >> p[2];
            verts.push_back(p);
        }
        else if (tag == "f")
        {
            std::vector<int> idx;
            std::string tok;
            while (ss >> tok)
            {
                int k = std::atoi(tok.substr(0, tok.find('/')).c_str());
                if (k < 0)
                    k = (int)verts.size() + k;
                else
                    k = k - 1;
                idx.push_back(k);
            }
            for (size_t j = 2; j < idx.size(); j++)  // fan triangulation of polygons
                tris.push_back({idx[0], idx[j - 1], idx[j]});
        }
    }
    for (auto &t : tris)
        for (int k : t)
            if (k < 0 || k >= (int)verts.size())
            {
                err = "face index out of range in " + path;
                return false;
            }
    if (tris.empty())
    {
        err = "no triangles in " + path;
        return false;
    }
    return true;
}

// ------------------------------------------------------------------ boxes ----------------
void BBox::add(const Vec3 &p)
{
    for (int k = 0; k < 3; k++)
    {
        lo[k] = std::min(lo[k], p[k]);
        hi[k] = std::max(hi[k], p[k]);
    }
}

void BBox::add(const BBox &b)
{
    add(b.lo);
    add(b.hi);
}

Vec3 BBox::center() const { return {(lo[0] + hi[0]) / 2, (lo[1] + hi[1]) / 2, (lo[2] + hi[2]) / 2}; }

float BBox::length() const { return std::max(std::max(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]); }

// ------------------------------------------------------------------ objects --------------
ManualObject::ManualObject(const Mesh &m)
{
    verts = m.verts;
    tris = m.tris;
}

void ManualObject::submit_acc(float *dst) const { std::fill(dst, dst + tris.size(), 0.0f); }

BBox ManualObject::bbox() const
{
    BBox b;
    for (auto &p : verts)
        b.add(p);
    return b;
}

namespace
{
// v' = 2 (u.v) u + (s^2 - u.u) v + 2 s (u x v), q = (u, s) not normalised (Object.cu:6-11)
Vec3 rotate(const std::array<float, 4> &q, const Vec3 &v)
{
    float ux = q[0], uy = q[1], uz = q[2], s = q[3];
    float uv = ux * v[0] + uy * v[1] + uz * v[2];
    float uu = ux * ux + uy * uy + uz * uz;
    Vec3 c{uy * v[2] - uz * v[1], uz * v[0] - ux * v[2], ux * v[1] - uy * v[0]};
    Vec3 r;
    for (int k = 0; k < 3; k++)
    {
        float u = k == 0 ? ux : (k == 1 ? uy : uz);
        r[k] = 2.0f * uv * u + (s * s - uu) * v[k] + 2.0f * s * c[k];
    }
    return r;
}
}  // namespace

bool AudioObject::load(const std::string &dir, std::string &err)
{
    Mesh m;
    if (!m.load_obj(dir + "/mesh.obj", err))
        return false;
    verts = standard = m.verts;
    tris = m.tris;
    {
        std::ifstream in(dir + "/motion.txt");
        std::string line;
        while (in.good() && std::getline(in, line))
        {
            if (line.empty())
                continue;
            std::istringstream ss(line);
            float t;
            Vec3 tr;
            std::array<float, 4> q;
            ss >> t >> tr[0] >> tr[1] >> tr[2] >> q[0] >> q[1] >> q[2] >> q[3];
            frame_time.push_back(t);
            translations.push_back(tr);
            rotations.push_back(q);
        }
    }
    {
        std::ifstream in(dir + "/accs.txt");
        float a;
        while (in.good() && (in >> a))
            accs.push_back(a);
    }
    selected.assign(tris.size(), 0);
    std::ifstream sel(dir + "/selected_vertices.txt");
    if (!sel.good())
        std::fill(selected.begin(), selected.end(), 1);  // every triangle carries the acceleration
    else
    {
        // the reference appends the value of the failing read at end of file too
        // (Object.cu:255-266), so vertex 0 joins the selection
        std::vector<int> cover;
        while (true)
        {
            int v = 0;
            sel >> v;
            cover.push_back(sel.fail() ? 0 : v);
            if (!sel.good())
                break;
        }
        for (int v : cover)
        {
            int face = -1;
            for (size_t f = 0; f < tris.size() && face < 0; f++)
                if (tris[f][0] == v || tris[f][1] == v || tris[f][2] == v)
                    face = (int)f;
            if (face >= 0)
                selected[face]++;
        }
    }
    return true;
}

void AudioObject::transform(int frame)
{
    for (size_t i = 0; i < verts.size(); i++)
    {
        Vec3 r = rotate(rotations[frame], standard[i]);
        for (int k = 0; k < 3; k++)
            verts[i][k] = r[k] + translations[frame][k];
    }
}

// Object.h:288-317: advance motion frames with frame time <= t, then the acceleration sample
bool AudioObject::update_until(float time)
{
    bool moved = false;
    if (anim_step + 1 < (int)frame_time.size())
    {
        while (anim_step + 1 < (int)frame_time.size() && frame_time[anim_step + 1] <= time)
        {
            anim_step++;
            moved = true;
        }
        if (moved)
            transform(anim_step);
    }
    acc_step++;
    while (sample_time * acc_step <= time)
        acc_step++;
    acc_step--;
    return moved;
}

void AudioObject::submit_acc(float *dst) const
{
    if (acc_step >= (int)accs.size())
    {
        std::fill(dst, dst + tris.size(), 0.0f);
        return;
    }
    for (size_t f = 0; f < tris.size(); f++)
        dst[f] = selected[f] > 0 ? accs[acc_step] : 0.0f;
}

BBox AudioObject::bbox() const
{
    BBox b;
    if (translations.empty())
    {
        for (auto &p : verts)
            b.add(p);
        return b;
    }
    for (size_t fr = 0; fr < translations.size(); fr++)
        for (auto &p : standard)
        {
            Vec3 r = rotate(rotations[fr], p);
            b.add(Vec3{r[0] + translations[fr][0], r[1] + translations[fr][1], r[2] + translations[fr][2]});
        }
    return b;
}

void AudioObject::save_state()
{
    saved.verts = verts;
    saved.anim_step = anim_step;
    saved.acc_step = acc_step;
}

void AudioObject::load_state()
{
    verts = saved.verts;
    anim_step = saved.anim_step;
    acc_step = saved.acc_step;
}

// ------------------------------------------------------------------ collection -----------
bool Collection::load(const std::string &root, const SceneConfig &cfg, std::string &err)
{
    for (auto &info : cfg.objects)
    {
        auto nit = info.find("name"), tit = info.find("type");
        if (nit == info.end() || tit == info.end())
        {
            err = "object entry needs name and type";
            return false;
        }
        std::string dir = root + "/" + nit->second;
        if (tit->second == "Audio")
        {
            auto o = std::make_unique<AudioObject>();
            if (!o->load(dir, err))
                return false;
            o->name = nit->second;
            objects.push_back(std::move(o));
        }
        else if (tit->second == "Manual")
        {
            Mesh m;
            if (!m.load_obj(dir + "/mesh.obj", err))
                return false;
            auto o = std::make_unique<ManualObject>(m);
            o->name = nit->second;
            objects.push_back(std::move(o));
        }
        else
        {
            err = "unsupported object type: " + tit->second + " (Audio and Manual are supported)";
            return false;
        }
    }
    if (objects.empty())
    {
        err = "no objects in the scene";
        return false;
    }
    return true;
}

BBox Collection::bbox() const
{
    BBox b;
    for (auto &o : objects)
        b.add(o->bbox());
    return b;
}

int Collection::n_verts() const
{
    int n = 0;
    for (auto &o : objects)
        n += (int)o->verts.size();
    return n;
}

int Collection::n_tris() const
{
    int n = 0;
    for (auto &o : objects)
        n += (int)o->tris.size();
    return n;
}

void Collection::gather_verts(std::vector<float> &out) const
{
    out.clear();
    for (auto &o : objects)
        for (auto &p : o->verts)
            out.insert(out.end(), p.begin(), p.end());
}

void Collection::gather_tris(std::vector<int> &out) const
{
    out.clear();
    int off = 0;
    for (auto &o : objects)
    {
        for (auto &t : o->tris)
            for (int k : t)
                out.push_back(k + off);
        off += (int)o->verts.size();
    }
}

void Collection::gather_acc(std::vector<float> &out) const
{
    out.assign(n_tris(), 0.0f);
    size_t off = 0;
    for (auto &o : objects)
    {
        o->submit_acc(out.data() + off);
        off += o->tris.size();
    }
}

}  // namespace pppm_host
