// Scene host of libpppm_b200: the reference's scene/config interface, re-implemented in C++
// on top of the C ABI.
//
//   SceneConfig    the line-oriented json-like config (src/utils/simple_json_reader.h:16-85):
//                  line 1 "{", two directory lines, numeric "key: value" lines up to a line
//                  holding '[', then per object a "{" line, two key lines, a "}" line, until ']'.
//                  Missing numeric keys read as 0, like std::map::operator[].
//   Mesh           Wavefront OBJ triangles (v / f records; 1-based or negative indices).
//   ManualObject   static mesh, silent (src/utils/Object.h:75-128).
//   AudioObject    mesh.obj + motion.txt (time tx ty tz qx qy qz qw) + accs.txt (one scalar per
//                  44.1 kHz sample) + optional selected_vertices.txt (Object.h:130-321):
//                  motion frames applied when frame time <= t with the unnormalised quaternion
//                  rotation of Object.cu:6-11, accelerations held per sample, filled into the
//                  selected triangles.
//   Collection     objects concatenated into one triangle soup in config order
//                  (src/utils/ObjectCollection.cu:21-207).
#pragma once
#include <array>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace pppm_host
{

using Vec3 = std::array<float, 3>;

struct SceneConfig
{
    std::map<std::string, std::string> dirs;
    std::map<std::string, float> nums;
    std::vector<std::map<std::string, std::string>> objects;
    bool load(const std::string &path, std::string &err);
    float num(const std::string &key) const;  // 0 when absent
};

struct Mesh
{
    std::vector<Vec3> verts;
    std::vector<std::array<int, 3>> tris;
    bool load_obj(const std::string &path, std::string &err);
};

struct BBox
{
    Vec3 lo{1e10f, 1e10f, 1e10f};
    Vec3 hi{-1e10f, -1e10f, -1e10f};
    void add(const Vec3 &p);
    void add(const BBox &b);
    Vec3 center() const;
    float length() const;  // longest side
};

class Object
{
  public:
    virtual ~Object() = default;
    virtual bool update_until(float time) = 0;  // true when the mesh moved
    virtual void submit_acc(float *dst) const = 0;
    virtual BBox bbox() const = 0;
    virtual void save_state() = 0;
    virtual void load_state() = 0;
    std::vector<Vec3> verts;
    std::vector<std::array<int, 3>> tris;
    std::string name;
};

class ManualObject : public Object
{
  public:
    explicit ManualObject(const Mesh &m);
    bool update_until(float) override { return false; }
    void submit_acc(float *dst) const override;
    BBox bbox() const override;
    void save_state() override {}
    void load_state() override {}
};

class AudioObject : public Object
{
  public:
    bool load(const std::string &dir, std::string &err);
    bool update_until(float time) override;
    void submit_acc(float *dst) const override;
    BBox bbox() const override;
    void save_state() override;
    void load_state() override;
    float sample_time = 1.0f / 44100.0f;

  private:
    void transform(int frame);
    std::vector<Vec3> standard;
    std::vector<Vec3> translations;
    std::vector<std::array<float, 4>> rotations;
    std::vector<float> frame_time;
    std::vector<float> accs;
    std::vector<int> selected;  // per triangle: number of selected vertices mapped to it
    int anim_step = -1;
    int acc_step = 0;
    struct
    {
        std::vector<Vec3> verts;
        int anim_step, acc_step;
    } saved;
};

class Collection
{
  public:
    bool load(const std::string &root, const SceneConfig &cfg, std::string &err);
    BBox bbox() const;
    void gather_verts(std::vector<float> &out) const;  // concatenated xyz
    void gather_tris(std::vector<int> &out) const;     // concatenated, offset indices
    void gather_acc(std::vector<float> &out) const;
    int n_verts() const;
    int n_tris() const;
    std::vector<std::unique_ptr<Object>> objects;
};

}  // namespace pppm_host
