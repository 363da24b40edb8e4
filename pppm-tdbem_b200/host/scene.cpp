// Scene host: config reader, OBJ loader, Audio / Manual objects, object collection.
#include "scene.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <unordered_map>

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

namespace
{
// motion.txt: "time tx ty tz qx qy qz qw" per frame (Object.cu: LoadMotion_)
void load_motion(const std::string &path, std::vector<float> &frame_time, std::vector<Vec3> &translations,
                 std::vector<std::array<float, 4>> &rotations)
{
    std::ifstream in(path);
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
}  // namespace

bool AudioObject::load(const std::string &dir, std::string &err)
{
    Mesh m;
    if (!m.load_obj(dir + "/mesh.obj", err))
        return false;
    verts = standard = m.verts;
    tris = m.tris;
    load_motion(dir + "/motion.txt", frame_time, translations, rotations);
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


// ------------------------------------------------------------------ modal objects --------
// Rayleigh damping per material (src/utils/material.h); unknown names give no damping
bool Material::set(const std::string &name)
{
    static const struct
    {
        const char *name;
        float alpha, beta;
    } table[] = {{"ceramic", 40.0f, 1e-7f}, {"plastic", 30.0f, 1e-6f}, {"steel", 5.0f, 3e-8f},
                 {"mdf", 35.0f, 5e-6f},     {"wood", 60.0f, 2e-6f}};
    for (auto &m : table)
        if (name == m.name)
        {
            alpha = m.alpha;
            beta = m.beta;
            return true;
        }
    alpha = beta = 0.0f;
    return false;
}

namespace
{
// Boundary faces of a tet mesh: faces that belong to one tet only, wound so that the normal points
// away from that tet's fourth vertex (Object.cu: FindAllSurfaces).  The faces are visited in the
// iteration order of a hash map keyed by the sorted vertex triple with the reference's hash, so
// the face order (and with it the triangle numbering of the scene) is the reference's.
struct TriKeyHash
{
    size_t operator()(const std::array<int, 3> &k) const
    {
        unsigned u = ((unsigned)k[0] << 20) + ((unsigned)k[1] << 10) + (unsigned)k[2];
        return (size_t)(long long)(int)u;  // an int hash widened as the reference's is
    }
};

void boundary_faces(const std::vector<std::array<int, 4>> &tets, const std::vector<Vec3> &v,
                    std::vector<std::array<int, 3>> &faces, std::vector<Vec3> &normals)
{
    struct Info
    {
        int cnt = 0, tet = 0, except = 0;
    };
    std::unordered_map<std::array<int, 3>, Info, TriKeyHash> cand;
    for (int i = 0; i < (int)tets.size(); i++)
        for (int i0 = 0; i0 < 4; i0++)
        {
            std::array<int, 3> tri;
            for (int j = 0, k = 0; j < 4; j++)
                if (j != i0)
                    tri[k++] = tets[i][j];
            Info &in = cand[tri];
            in.cnt++;
            in.tet = i;
            in.except = i0;
        }
    for (auto &kv : cand)
    {
        if (kv.second.cnt != 1)
            continue;
        std::array<int, 3> t = kv.first;
        const Vec3 &a = v[t[0]], &b = v[t[1]], &c = v[t[2]];
        Vec3 centre, ex, e1, e2, n;
        for (int k = 0; k < 3; k++)
        {
            centre[k] = (a[k] + b[k] + c[k]) / 3;
            e1[k] = b[k] - a[k];
            e2[k] = c[k] - a[k];
        }
        const Vec3 &far = v[tets[kv.second.tet][kv.second.except]];
        for (int k = 0; k < 3; k++)
            ex[k] = far[k] - centre[k];
        n = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        float inv = 1.0f / std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (int k = 0; k < 3; k++)
            n[k] *= inv;
        if (n[0] * ex[0] + n[1] * ex[1] + n[2] * ex[2] > 0)
        {
            std::swap(t[1], t[2]);
            for (int k = 0; k < 3; k++)
                n[k] = -n[k];
        }
        faces.push_back(t);
        normals.push_back(n);
    }
}
}  // namespace

bool ModalObject::load(const std::string &dir, const std::string &material_name, std::string &err,
                       float max_frequency)
{
    material.set(material_name);
    load_motion(dir + "/motion.txt", frame_time, translations, rotations);
    {
        std::ifstream in(dir + "/contact.txt");
        if (!in.good())
        {
            err = "cannot read " + dir + "/contact.txt";
            return false;
        }
        std::string line;
        while (std::getline(in, line))
        {
            if (line.empty())
                continue;
            std::istringstream ss(line);
            float t, vid, nx, ny, nz, mag;
            ss >> t >> vid >> nx >> ny >> nz >> mag;
            impulses.push_back({t, (int)(vid + 0.5f), Vec3{nx * mag, ny * mag, nz * mag}});
        }
    }
    {
        std::ifstream in(dir + "/vertices.txt");
        if (!in.good())
        {
            err = "cannot read " + dir + "/vertices.txt";
            return false;
        }
        std::string line;
        while (std::getline(in, line))
        {
            if (line.empty())
                continue;
            std::istringstream ss(line);
            Vec3 p;
            ss >> p[0] >> p[1] >> p[2];
            standard.push_back(p);
        }
    }
    std::vector<std::array<int, 4>> tets;
    {
        std::ifstream in(dir + "/tets.txt");
        if (!in.good())
        {
            err = "cannot read " + dir + "/tets.txt";
            return false;
        }
        std::string line;
        while (std::getline(in, line))
        {
            if (line.empty())
                continue;
            std::istringstream ss(line);
            float f[4];
            ss >> f[0] >> f[1] >> f[2] >> f[3];
            std::array<int, 4> t;
            for (int k = 0; k < 4; k++)
                t[k] = (int)(f[k] + 0.5f);
            std::sort(t.begin(), t.end());
            for (int k = 0; k < 4; k++)
                if (t[k] < 0 || t[k] >= (int)standard.size())
                {
                    err = "tet vertex index out of range in " + dir + "/tets.txt";
                    return false;
                }
            tets.push_back(t);
        }
    }
    boundary_faces(tets, standard, tris, normals);
    verts = standard;
    // eigenvalues ascending; modes below max_frequency kept (RigidBody.cu: LoadEigen_)
    std::vector<float> all;
    {
        std::ifstream in(dir + "/eigenvalues.txt");
        if (!in.good())
        {
            err = "cannot read " + dir + "/eigenvalues.txt";
            return false;
        }
        std::string line;
        int keep = 0;
        while (std::getline(in, line))
        {
            if (line.empty())
                continue;
            std::istringstream ss(line);
            float val;
            ss >> val;
            all.push_back(val);
            if (std::sqrt(val) / (2 * M_PI) < max_frequency)
                keep = (int)all.size();
        }
        eigen.assign(all.begin(), all.begin() + keep);
    }
    const int dim = 3 * (int)standard.size(), nm = (int)eigen.size();
    vecs.assign((size_t)dim * nm, 0.0f);
    {
        std::ifstream in(dir + "/eigenvectors.txt");
        if (!in.good())
        {
            err = "cannot read " + dir + "/eigenvectors.txt";
            return false;
        }
        for (int i = 0; i < dim; i++)
            for (int j = 0; j < (int)all.size(); j++)
            {
                float val = 0;
                in >> val;
                if (j < nm)
                    vecs[(size_t)i * nm + j] = val;
            }
        if (in.fail())
        {
            err = "eigenvectors.txt holds fewer than 3 x vertices x eigenvalues values";
            return false;
        }
    }
    // per face: normal . mean of its vertices' mode shapes (RigidBody.cu: MatrixVertToTri)
    surf.assign(tris.size() * (size_t)nm, 0.0f);
    for (size_t f = 0; f < tris.size(); f++)
        for (int i = 0; i < nm; i++)
        {
            float m[3];
            for (int k = 0; k < 3; k++)
                m[k] = (vecs[(size_t)(3 * tris[f][0] + k) * nm + i] + vecs[(size_t)(3 * tris[f][1] + k) * nm + i] +
                        vecs[(size_t)(3 * tris[f][2] + k) * nm + i]) /
                       3;
            surf[f * nm + i] = m[0] * normals[f][0] + m[1] * normals[f][1] + m[2] * normals[f][2];
        }
    accs.assign(tris.size(), 0.0f);
    return true;
}

// IIR coefficients of one damped mode (RigidBody.cu: ModalInfo::SetCoeffs), in float
void ModalObject::set_sample_rate(float rate)
{
    timestep = 1.0f / rate;
    modes.assign(eigen.size(), Mode{});
    for (size_t i = 0; i < eigen.size(); i++)
    {
        float lambda = eigen[i];
        float omega = std::sqrt(lambda);
        float ksi = (material.alpha + material.beta * lambda) / (2 * omega);
        float omega_d = omega * std::sqrt(1 - ksi * ksi);
        float eps = std::exp(-ksi * omega * timestep);
        float eps2 = eps * eps;
        float theta = omega_d * timestep;
        float gamma = std::asin(ksi);
        Mode &m = modes[i];
        m.c1 = 2 * eps * std::cos(theta);
        m.c2 = -eps2;
        float a = eps * std::cos(theta + gamma);
        float b = eps2 * std::cos(2 * theta + gamma);
        m.c3 = 2 * (a - b) / (3 * omega * omega_d);
    }
    active.clear();
    current_time = 0;
    anim_step = 0;
}

void ModalObject::transform(int frame)
{
    for (size_t i = 0; i < verts.size(); i++)
    {
        Vec3 r = rotate(rotations[frame], standard[i]);
        for (int k = 0; k < 3; k++)
            verts[i][k] = r[k] + translations[frame][k];
    }
}

// one audio sample (RigidBody.cu: audio_step, CalculateIIR_): the motion frame due, then the
// contact forces of the impulses active at the new time (half sines of 0.5 ms), the modal IIR
// step and the faces' accelerations
void ModalObject::audio_step()
{
    moved_ = false;
    if (anim_step < (int)frame_time.size() && frame_time[anim_step] <= current_time)
    {
        transform(anim_step);
        anim_step++;
        moved_ = true;
    }
    current_time += timestep;
    const float now = current_time, tau = 0.0005f;
    while (impulse_step < (int)impulses.size() && now >= impulses[impulse_step].time)
        active.push_back(impulses[impulse_step++]);
    while (!active.empty() && now - active.front().time > tau)
        active.erase(active.begin());
    const int nm = (int)modes.size();
    std::vector<float> qdd(nm);
    for (int i = 0; i < nm; i++)
    {
        Mode &m = modes[i];
        m.f = 0;
        for (auto &imp : active)
        {
            const float amp = (float)std::sin(M_PI * (now - imp.time) / tau);
            const float jx = imp.vec[0] * amp, jy = imp.vec[1] * amp, jz = imp.vec[2] * amp;
            const size_t r = (size_t)imp.vertex * 3;
            m.f += vecs[r * nm + i] * jx + vecs[(r + 1) * nm + i] * jy + vecs[(r + 2) * nm + i] * jz;
        }
        const float q0 = m.c1 * m.q1 + m.c2 * m.q2 + m.c3 * m.f;
        m.q3 = m.q2;
        m.q2 = m.q1;
        m.q1 = q0;
        qdd[i] = (m.q1 + m.q3 - 2 * m.q2) / (timestep * timestep);
    }
    for (size_t f = 0; f < tris.size(); f++)
    {
        float a = 0;
        for (int i = 0; i < nm; i++)
            a += surf[f * nm + i] * qdd[i];
        accs[f] = a;
    }
}

bool ModalObject::update_until(float time)
{
    bool moved = false;
    while (current_time < time)
    {
        audio_step();
        moved = moved_;
    }
    return moved;
}

void ModalObject::move_to_first_impulse()
{
    if (impulses.empty() || timestep <= 0)
        return;
    while (current_time + timestep < impulses[0].time)
        audio_step();
}

void ModalObject::submit_acc(float *dst) const { std::copy(accs.begin(), accs.end(), dst); }

BBox ModalObject::bbox() const
{
    BBox b;
    if (translations.empty())
    {
        for (auto &p : verts)
            b.add(p);
        return b;
    }
    // motion frames from the one in force at the first contact on (RigidBody.cu: get_bbox)
    size_t t = 1;
    if (!impulses.empty())
        while (t < frame_time.size() && frame_time[t] < impulses[0].time)
            t++;
    t = t > 0 ? t - 1 : 0;
    for (; t < translations.size(); t++)
        for (auto &p : standard)
        {
            Vec3 r = rotate(rotations[t], p);
            b.add(Vec3{r[0] + translations[t][0], r[1] + translations[t][1], r[2] + translations[t][2]});
        }
    return b;
}

// the reference's saved state: vertices, modal IIR state, face accelerations, time stamps and time
// (the list of active impulses is not part of it)
void ModalObject::save_state()
{
    saved.verts = verts;
    saved.modes = modes;
    saved.accs = accs;
    saved.anim_step = anim_step;
    saved.impulse_step = impulse_step;
    saved.current_time = current_time;
}

void ModalObject::load_state()
{
    verts = saved.verts;
    modes = saved.modes;
    accs = saved.accs;
    anim_step = saved.anim_step;
    impulse_step = saved.impulse_step;
    current_time = saved.current_time;
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
        else if (tit->second == "Modal")
        {
            // the demo driver builds every Modal object with the "plastic" material
            // (experiments/demo/main.cu:62-66)
            auto o = std::make_unique<ModalObject>();
            if (!o->load(dir, "plastic", err))
                return false;
            o->name = nit->second;
            modal.push_back(o.get());
            objects.push_back(std::move(o));
        }
        else
        {
            err = "unsupported object type: " + tit->second + " (Audio, Manual and Modal are supported)";
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
