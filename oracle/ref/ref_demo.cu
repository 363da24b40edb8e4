// Headless driver of the reference's scene layer and solver (TEST INFRASTRUCTURE: built into
// oracle/_ref/ref_demo from the reference's own sources by oracle/Makefile, run only by the GPU
// parity tests of the scene host).
//
//     ref_demo CONFIG
//
// Runs a scene config through the reference's own classes - SimpleJsonReader
// (src/utils/simple_json_reader.h), ObjectCollection with Audio / Manual / Modal objects
// (src/utils/ObjectCollection.cu, Object.h/.cu, RigidBody.cu) and PPPMSolver (src/algorithm/pppm.h) -
// in the order of the demo driver's AudioAndManualTest (experiments/demo/main.cu:38-275), and
// writes outputDir/result.txt.  Left out, because they need what this machine has not: the GL /
// imgui window and PNG dumps (main.cu:4-10, 22-36), the pymesh docker repair (replaced by the
// identity repair of shim/identity_fix_mesh.h: the test meshes are clean), the water-muting hack
// (main.cu:49-72).  Everything that decides result.txt is the reference's: grid placement, frame
// rate, the Modal objects' lead-in, the per-step object updates, the chunked cross-fade restart
// and the listener read.
#include <algorithm>
#include <any>
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <string>
#include <utility>
#include <vector>

#include "ObjectCollection.h"
#include "RigidBody.h"
#include "array_writer.h"
#include "pppm.h"
#include "simple_json_reader.h"

using namespace pppm;

namespace
{
struct Scene
{
    SimpleJsonReader cfg;
    std::vector<std::pair<std::string, ObjectInfo::SoundType>> names;
    std::vector<std::any> extra;
    explicit Scene(const char *path) : cfg(path) {}
    float num(const char *key) { return cfg.numMap[key]; }  // absent keys read 0, as in the reference
};

std::vector<RigidBody *> modal_objects(ObjectCollection &col)
{
    std::vector<RigidBody *> out;
    for (size_t i = 0; i < col.objectInfos.size(); i++)
        if (col.objectInfos[i].type == ObjectInfo::SoundType::Modal)
            out.push_back(static_cast<RigidBody *>(col.objects[i].get()));
    return out;
}
}  // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
    {
        std::fprintf(stderr, "usage: ref_demo CONFIG\n");
        return 2;
    }
    Scene sc(argv[1]);
    const std::string in_dir = sc.cfg.dirMap["inputDir"], out_dir = sc.cfg.dirMap["outputDir"];
    std::filesystem::create_directories(out_dir);
    for (auto &info : sc.cfg.sceneInfoMap)
    {
        const std::string &type = info["type"];
        if (info["name"] == "water")
        {
            std::fprintf(stderr, "ref_demo: the water-muting scene is not supported\n");
            return 2;
        }
        if (type == "Audio")
        {
            sc.names.emplace_back(info["name"], ObjectInfo::SoundType::Audio);
            sc.extra.emplace_back();
        }
        else if (type == "Manual")
        {
            sc.names.emplace_back(info["name"], ObjectInfo::SoundType::Manual);
            sc.extra.emplace_back();
        }
        else if (type == "Modal")
        {
            sc.names.emplace_back(info["name"], ObjectInfo::SoundType::Modal);
            sc.extra.emplace_back(std::string{"plastic"});
        }
        else
        {
            std::fprintf(stderr, "ref_demo: unknown sound type %s\n", type.c_str());
            return 2;
        }
    }
    ObjectCollection col(in_dir, sc.names, sc.extra);

    // grid around the scene's bounding box over the whole motion (main.cu:96-103)
    BBox box = col.GetBBox();
    const float length = box.length() * sc.num("gridLengthFactor");
    const int res = sc.num("res");
    const float h = length / res;
    const float3 min_pos = box.center() - length / 2;
    const int rate = 1.01f / (h / std::sqrt(3) / AIR_WAVE_SPEED);
    for (RigidBody *rb : modal_objects(col))
        rb->set_sample_rate(rate);
    col.UpdateTimeStep();
    col.FixMesh(h);
    // the run starts at the first contact of the modal objects; the steps before it are silent
    float now = 0;
    for (RigidBody *rb : modal_objects(col))
    {
        rb->move_to_first_impulse();
        now = std::max(now, rb->current_time);
    }
    const int silent = now * rate;
    col.UpdateMesh();
    const float dt = 1.0f / rate;
    now += sc.num("startTime");
    const float end = sc.num("maxTime") + now;
    PPPMSolver solver(res, h, dt, min_pos, 0, sc.num("reflectCoeff"));
    const int nframes = (end - now) / dt;
    const int3 listener = make_int3(sc.num("checkCoordX") * res, sc.num("checkCoordY") * res,
                                    sc.num("checkCoordZ") * res);
    CArr<float> result(silent + nframes + 2);
    result.reset();
    result[0] = rate;
    const int chunk = sc.num("chunkSize"), back = sc.num("backStepSize");
    if (chunk <= 0)
    {
        std::fprintf(stderr, "ref_demo: chunkSize must be positive (the reference divides by it)\n");
        return 2;
    }

    // one step of the scene: objects to the end of the step (a step in which one object's mesh
    // moved skips the updates of the objects after it, as the reference's || does), gathered
    // surface, accelerations (zero when muted), solver mesh and step
    auto advance = [&](bool muted) {
        bool moved = false;
        for (auto &obj : col.objects)
            moved = moved || obj->UpdateUntil(now + dt);
        now += dt;
        col.UpdateMesh();
        col.UpdateAcc();
        if (!solver.mesh_set)
            solver.set_mesh(col.tetVertices, col.tetSurfaces);
        else if (moved)
            solver.update_mesh(col.tetVertices);
        if (muted)
            col.surfaceAccs.reset();
        solver.update_grid_and_face(col.surfaceAccs);
    };
    auto sample = [&]() { return solver.pg.fdtd.grids[solver.pg.fdtd.t](to_cpu(listener)); };

    int step = 0;
    while (step <= nframes)
    {
        const int i = step;
        if (i % chunk == chunk - back)
        {
            // cross-fade restart: the rest of the chunk once muted and fading out, then again from
            // the saved time with fresh fields, added (main.cu:212-263)
            const int last = std::min<int>(i + back, nframes + 1);
            const int saved_t = solver.pg.fdtd.t;
            const float saved_now = now;
            for (size_t k = 0; k < col.objects.size(); k++)
                col.objects[k]->SaveState(*(col.objectInfos[k].state));
            for (int j = i; j < last; j++)
            {
                advance(true);
                const float fade = (float)(j - i) / (float)(last - i);
                result[silent + j + 1] = sample() * (1 - fade);
            }
            solver.pg.fdtd.reset();
            solver.neumann.reset();
            solver.dirichlet.reset();
            solver.pg.fdtd.t = saved_t;
            now = saved_now;
            for (size_t k = 0; k < col.objects.size(); k++)
                col.objects[k]->LoadState(*(col.objectInfos[k].state));
            for (int j = i; j < last; j++)
            {
                advance(false);
                result[silent + j + 1] += sample();
                step++;
            }
            continue;
        }
        advance(false);
        result[silent + i + 1] = sample();
        step++;
    }
    write_to_txt(out_dir + "/result.txt", result);
    solver.clear();
    return 0;
}
