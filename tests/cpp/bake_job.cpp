// A full-scene bake through Relight::bake, shaped like Relight's demo
// (src/demo/Lightmapping.cpp:270-297): photons first, then a Job whose
// execute() bakes direct and indirect light for the JobData's mesh and
// iterator, pushed by Relight::bake's FullBakeJob to every worker for every
// mesh of the scene.
//
//   bake_job <out-prefix>
//     <out-prefix>.workers.bin   3 base Workers (jobs run on the calling
//                                thread): direct + final gather
//     <out-prefix>.threads.bin   4 thread workers (one std::thread per push,
//                                as the demo's ThreadWorker): direct light only
// Each file holds the lightmap's flags, then its RGB colours.
#include "room_scene.h"

#include <thread>

using namespace relight;
using namespace room_example;

struct Bake : public Job {
    Bake(const IndirectLightSettings& indirect, bool indirectToo) : m_indirect(indirect), m_both(indirectToo) {}
    void execute(JobData* data) override {
        data->m_relight->bakeDirectLight(data->m_scene, data->m_mesh, data->m_worker, data->m_iterator);
        if (m_both)
            data->m_relight->bakeIndirectLight(data->m_scene, data->m_mesh, data->m_worker, m_indirect,
                                               data->m_iterator);
        m_calls++;
    }
    IndirectLightSettings m_indirect;
    bool m_both;
    int m_calls = 0;
};

// The demo's ThreadWorker: each push starts a thread that runs the job and
// frees its JobData; wait() joins it.
struct ThreadWorker : public Worker {
    void push(Job* job, JobData* data) override {
        data->m_worker = this;
        m_thread = std::thread([job, data]() {
            job->execute(data);
            delete data;
        });
    }
    void wait() override {
        if (m_thread.joinable()) m_thread.join();
    }
    void notify(const Mesh*, int, int) override { m_notified++; }
    std::thread m_thread;
    int m_notified = 0;
};

int main(int argc, char** argv) {
    std::string out = argc > 1 ? argv[1] : "bake_job";
    IndirectLightSettings ind = IndirectLightSettings::draft(Rgb(0.2f, 0.2f, 0.3f), Rgb(0, 0, 0), 20.0f, 20.0f);
    ind.m_photonPassCount = 1;
    ind.m_finalGatherSamples = 16;

    {
        RoomScene rs;
        if (!build_room(rs)) return 2;
        if (rs.relight->emitPhotons(rs.scene, ind) != RelightSuccess) return 3;
        Bake job(ind, true);
        Worker root;
        Workers workers;
        for (int i = 0; i < 3; i++) workers.push_back(new Worker);
        rs.relight->bake(rs.scene, &job, &root, workers);
        // 2 meshes x 3 workers
        if (job.m_calls != 6) return 4;
        if (!dump(rs.lightmap, out + ".workers.bin")) return 5;
        for (Worker* w : workers) delete w;
    }
    {
        RoomScene rs;
        if (!build_room(rs)) return 6;
        Bake job(ind, false);
        ThreadWorker root;
        std::vector<ThreadWorker*> threads;
        Workers workers;
        for (int i = 0; i < 4; i++) {
            threads.push_back(new ThreadWorker);
            workers.push_back(threads.back());
        }
        rs.relight->bake(rs.scene, &job, &root, workers);
        root.wait();  // the root runs the FullBakeJob on its own thread
        if (job.m_calls != 8) return 7;
        for (ThreadWorker* t : threads)
            if (t->m_notified != 2) return 8;  // one bakeDirectLight per mesh
        if (!dump(rs.lightmap, out + ".threads.bin")) return 9;
        for (ThreadWorker* t : threads) delete t;
    }
    printf("bake_job ok: %s\n", out.c_str());
    return 0;
}
