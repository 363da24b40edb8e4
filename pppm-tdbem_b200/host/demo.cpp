// pppm_demo CONFIG - drop-in for the reference's `demo CONFIG` driver
// (experiments/demo/main.cu:38-282) on top of libpppm_b200's C ABI.
//
// Same scene semantics: grid centred on the scene's bounding box (all motion frames),
// length = gridLengthFactor * longest side, dt = 1 / int(1.01 / (h / sqrt(3) / 340.3)),
// listener at int(checkCoord * res), per step: objects advanced to t + dt (the first object
// that moves short-circuits the rest, as the reference's `moved = moved || update` does),
// set_mesh on the first step, update_mesh when a motion frame was applied, one time step with
// the gathered accelerations; every chunkSize steps the last backStepSize steps run twice
// (sources muted and faded out, then from zeroed fields and restored object states, added):
// the cross-fade restart of main.cu:212-263.  Output: outputDir/result.txt, line 0 the frame
// rate, then one "%e" sample per step.
//
// Modal objects (RigidBody): their IIR runs at the step rate; the run starts at the latest first
// contact, whose leading samples stay silent (zero) at the front of result.txt (main.cu:104-125,153).
//
// Differences, all where the reference is undefined or unavailable: no FixMesh (the reference
// shells out to a pymesh docker image); chunkSize <= 0 disables the cross-fade (the reference
// evaluates i % 0); a non-finite sample stops the run (the reference tests an index one past
// the sample it just wrote).  Steps between mesh updates are submitted to the device in one
// call and the listener samples read back once per batch instead of once per step.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "pppm_b200.h"
#include "scene.h"

using namespace pppm_host;

namespace
{

struct Pending
{
    int result_index;
    int mode;  // 0 assign, 1 add
    float factor;
};

class Runner
{
  public:
    pppm_handle *h = nullptr;
    int nt = 0;
    std::vector<float> rows;
    std::vector<Pending> pending;
    std::vector<float> *result = nullptr;
    int series_pos = 0;
    bool nan = false;

    int flush()
    {
        if (pending.empty())
            return PPPM_OK;
        int n = (int)pending.size();
        int rc = pppm_step(h, rows.data(), 0, n);
        if (rc)
            return rc;
        std::vector<float> out(n);
        rc = pppm_read_listeners(h, series_pos, n, out.data());
        if (rc && rc != PPPM_ERR_NAN)
            return rc;
        series_pos += n;
        for (int i = 0; i < n; i++)
        {
            if (!std::isfinite(out[i]))
                nan = true;
            float &dst = (*result)[pending[i].result_index];
            if (pending[i].mode == 0)
                dst = out[i] * pending[i].factor;
            else
                dst += out[i];
        }
        rows.clear();
        pending.clear();
        return PPPM_OK;
    }
};

int fail(const char *what, int rc)
{
    fprintf(stderr, "pppm_demo: %s failed: %s (%s)\n", what, pppm_status_string(rc), pppm_last_error_message());
    return 1;
}

}  // namespace

// pppm_demo --modal-accs DIR RATE NSAMPLES OUT: the surface accelerations of one Modal object
// (material "plastic") sampled at RATE from its first contact on, without the solver (the
// reference's RigidBody::export_surface_accs).  OUT: "faces modes time" on line 1, the faces'
// vertex triples, then one line of face accelerations per sample.
int export_modal(char **argv)
{
    ModalObject m;
    std::string err;
    if (!m.load(argv[2], "plastic", err))
    {
        fprintf(stderr, "pppm_demo: %s\n", err.c_str());
        return 1;
    }
    const float rate = (float)atof(argv[3]);
    const int n = atoi(argv[4]);
    if (!(rate > 0) || n < 0)
    {
        fprintf(stderr, "pppm_demo: bad RATE or NSAMPLES\n");
        return 2;
    }
    m.set_sample_rate(rate);
    m.move_to_first_impulse();
    FILE *f = fopen(argv[5], "w");
    if (!f)
    {
        fprintf(stderr, "pppm_demo: cannot write %s\n", argv[5]);
        return 1;
    }
    fprintf(f, "%zu %d %.9e\n", m.tris.size(), m.n_modes(), m.current_time);
    for (auto &t : m.tris)
        fprintf(f, "%d %d %d\n", t[0], t[1], t[2]);
    const float half = 0.5f / rate;
    for (int s = 0; s < n; s++)
    {
        m.update_until(m.current_time + half);  // one audio sample
        const auto &a = m.surface_acc();
        for (size_t k = 0; k < a.size(); k++)
            fprintf(f, k + 1 < a.size() ? "%.9e " : "%.9e\n", a[k]);
    }
    fclose(f);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc == 6 && std::strcmp(argv[1], "--modal-accs") == 0)
        return export_modal(argv);
    if (argc < 2)
    {
        fprintf(stderr, "usage: %s CONFIG\n       %s --modal-accs DIR RATE NSAMPLES OUT\n", argv[0], argv[0]);
        return 2;
    }
    SceneConfig cfg;
    std::string err;
    if (!cfg.load(argv[1], err))
    {
        fprintf(stderr, "pppm_demo: %s\n", err.c_str());
        return 1;
    }
    const std::string input = cfg.dirs["inputDir"], output = cfg.dirs["outputDir"];
    Collection col;
    if (!col.load(input, cfg, err))
    {
        fprintf(stderr, "pppm_demo: %s\n", err.c_str());
        return 1;
    }
    BBox bbox = col.bbox();
    Vec3 center = bbox.center();
    float grid_length = bbox.length() * cfg.num("gridLengthFactor");
    float reflect = cfg.num("reflectCoeff");
    int res = (int)cfg.num("res");
    if (res < 8 || !(grid_length > 0))
    {
        fprintf(stderr, "pppm_demo: res and gridLengthFactor must be set\n");
        return 1;
    }
    float grid_size = grid_length / res;
    float min_pos[3] = {center[0] - grid_length / 2, center[1] - grid_length / 2, center[2] - grid_length / 2};
    int frame_rate = (int)(1.01f / (grid_size / std::sqrt(3) / 340.3f));
    float dt = 1.0f / frame_rate;
    float curr_time = 0;
    // Modal objects: their IIR runs at the step rate, and the run starts at the latest first
    // contact, with that many leading samples left silent in the output (main.cu:104-125)
    for (ModalObject *m : col.modal)
        m->set_sample_rate((float)frame_rate);
    for (ModalObject *m : col.modal)
    {
        m->move_to_first_impulse();
        curr_time = std::max(curr_time, m->current_time);
    }
    const int mute_frames = (int)(curr_time * frame_rate);
    curr_time += cfg.num("startTime");
    float max_time = cfg.num("maxTime") + curr_time;
    int frame_num = (int)((max_time - curr_time) / dt);
    int check[3] = {(int)(cfg.num("checkCoordX") * res), (int)(cfg.num("checkCoordY") * res),
                    (int)(cfg.num("checkCoordZ") * res)};
    int chunk = (int)cfg.num("chunkSize"), back = (int)cfg.num("backStepSize");
    printf("res: %d\nmax time: %g\ngrid size: %g\ndt: %g\nframe rate: %d\ncheck_coord: %d %d %d\n", res, max_time,
           grid_size, dt, frame_rate, check[0], check[1], check[2]);

    pppm_params p;
    pppm_params_default(&p);
    p.res = res;
    p.dl = grid_size;
    p.dt = dt;
    for (int k = 0; k < 3; k++)
        p.min_pos[k] = min_pos[k];
    p.reflect_coeff = reflect;
    pppm_handle *h = nullptr;
    int rc = pppm_create(&p, &h);
    if (rc)
        return fail("pppm_create", rc);
    rc = pppm_add_listener(h, check[0], check[1], check[2]);
    if (rc)
        return fail("pppm_add_listener (checkCoord outside the grid?)", rc);

    std::vector<float> result(mute_frames + frame_num + 2, 0.0f);
    result[0] = (float)frame_rate;
    Runner run;
    run.h = h;
    run.nt = col.n_tris();
    run.result = &result;
    std::vector<float> verts, acc;
    std::vector<int> tris;
    col.gather_tris(tris);
    bool mesh_set = false;

    auto update_sound = [&](bool mute, int result_index, int mode, float factor) -> int {
        bool moved = false;
        for (auto &o : col.objects)
            moved = moved || o->update_until(curr_time + dt);
        curr_time += dt;
        if (!mesh_set || moved)
        {
            int r = run.flush();
            if (r)
                return r;
            col.gather_verts(verts);
            r = mesh_set ? pppm_update_mesh(h, verts.data(), 0)
                         : pppm_set_mesh(h, verts.data(), col.n_verts(), tris.data(), col.n_tris());
            if (r)
                return r;
            mesh_set = true;
        }
        if (mute)
            acc.assign(run.nt, 0.0f);
        else
            col.gather_acc(acc);
        run.rows.insert(run.rows.end(), acc.begin(), acc.end());
        run.pending.push_back({result_index, mode, factor});
        return PPPM_OK;
    };

    int progress = 0;
    while (progress <= frame_num && !run.nan)
    {
        int i = progress;
        if (chunk > 0 && i % chunk == chunk - back)
        {
            int end = std::min(i + back, frame_num + 1);
            if ((rc = run.flush()))
                return fail("step", rc);
            int saved_t = 0;
            pppm_get_time(h, &saved_t);
            float saved_time = curr_time;
            for (auto &o : col.objects)
                o->save_state();
            for (int j = i; j < end; j++)
                if ((rc = update_sound(true, mute_frames + j + 1, 0, 1.0f - (float)(j - i) / (float)(end - i))))
                    return fail("step", rc);
            if ((rc = run.flush()))
                return fail("step", rc);
            if (run.nan)
                break;
            pppm_reset_fields(h);
            pppm_set_time(h, saved_t);
            curr_time = saved_time;
            for (auto &o : col.objects)
                o->load_state();
            for (int j = i; j < end; j++)
                if ((rc = update_sound(false, mute_frames + j + 1, 1, 1.0f)))
                    return fail("step", rc);
            if ((rc = run.flush()))
                return fail("step", rc);
            progress += end - i;
            continue;
        }
        if ((rc = update_sound(false, mute_frames + i + 1, 0, 1.0f)))
            return fail("step", rc);
        progress++;
    }
    if ((rc = run.flush()))
        return fail("step", rc);
    if (run.nan)
        printf("NAN\n");
    printf("Done\n");
    std::error_code ec;
    std::filesystem::create_directories(output, ec);
    std::string path = output + "/result.txt";
    FILE *f = fopen(path.c_str(), "w");
    if (!f)
    {
        fprintf(stderr, "pppm_demo: cannot write %s\n", path.c_str());
        return 1;
    }
    for (size_t k = 0; k < result.size(); k++)
        fprintf(f, k + 1 < result.size() ? "%e\n" : "%e", result[k]);
    fclose(f);
    pppm_destroy(h);
    return 0;
}
