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
//   ModalObject    the reference's RigidBody ("Modal" type, src/utils/RigidBody.h/.cu): a tet mesh
//                  (vertices.txt, tets.txt) whose boundary faces are the sound surface, rigid
//                  motion (motion.txt), contact impulses (contact.txt: time vertex nx ny nz |J|)
//                  and its eigenmodes (eigenvalues.txt, eigenvectors.txt: 3 nv rows, one column
//                  per mode, modes up to 15 kHz kept).  Each audio sample advances one
//                  Rayleigh-damped modal IIR per mode (material "plastic", as the demo driver
//                  uses) driven by the impulses' half-sine contact forces; the surface
//                  acceleration of a face is its normal . (mean of its vertices' mode shapes)
//                  times the modal accelerations.  FixMesh (pymesh) is not done.  Boundary faces
//                  come in the reference's order (the iteration order of its hash map of face
//                  keys), so the scene's triangle numbering matches.
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

// material damping of the modal IIR (src/utils/material.h: Rayleigh alpha, beta per material)
struct Material
{
    float alpha = 0, beta = 0;
    bool set(const std::string &name);
};

class ModalObject : public Object
{
  public:
    bool load(const std::string &dir, const std::string &material, std::string &err, float max_frequency = 15000.0f);
    void set_sample_rate(float rate);  // the modal IIR runs at the solver's step rate
    void move_to_first_impulse();      // audio samples up to the first contact
    bool update_until(float time) override;
    void submit_acc(float *dst) const override;
    BBox bbox() const override;        // over the motion frames from the first contact on
    void save_state() override;
    void load_state() override;
    float current_time = 0;
    int n_modes() const { return (int)eigen.size(); }
    const std::vector<float> &surface_acc() const { return accs; }

  private:
    struct Impulse
    {
        float time;
        int vertex;
        Vec3 vec;  // normal * magnitude
    };
    struct Mode
    {
        float c1 = 0, c2 = 0, c3 = 0, f = 0, q1 = 0, q2 = 0, q3 = 0;
    };
    void audio_step();
    void transform(int frame);
    std::vector<Vec3> standard;
    std::vector<Vec3> normals;  // per surface face, of the rest shape
    std::vector<Vec3> translations;
    std::vector<std::array<float, 4>> rotations;
    std::vector<float> frame_time;
    std::vector<Impulse> impulses;
    std::vector<float> eigen;  // kept eigenvalues
    std::vector<float> vecs;   // (3 nv) x modes, row-major
    std::vector<float> surf;   // faces x modes
    std::vector<Mode> modes;
    std::vector<float> accs;   // per face
    std::vector<Impulse> active;
    Material material;
    float timestep = 0;
    int anim_step = 0, impulse_step = 0;
    bool moved_ = false;  // the last audio sample applied a motion frame
    struct
    {
        std::vector<Vec3> verts;
        std::vector<Mode> modes;
        std::vector<float> accs;
        int anim_step, impulse_step;
        float current_time;
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
    std::vector<ModalObject *> modal;  // the Modal objects among them
};

}  // namespace pppm_host
