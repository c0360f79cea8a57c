// GPU.cpp -- the GPU seam over libmpcf_b200 (see GPU.h).
#include "GPU.h"

#include <cstdio>
#include <cstdlib>

#include "../../include/mpcf_b200.h"

namespace
{
    mpcf_solver* g_current = nullptr;
    float g_last_sos = 0.0f;
}

namespace GPU
{
    mpcf_solver* current_solver() { return g_current; }
    void set_current_solver(mpcf_solver* s) { g_current = s; }
    float last_max_sos() { return g_last_sos; }
    void set_last_max_sos(float v) { g_last_sos = v; }

    void check(int rc, const char* what)
    {
        if (rc < 0)
        {
            fprintf(stderr, "[%s ERROR: %s]\n", what, mpcf_last_error());
            exit(1);
        }
    }

    static int current_device()
    {
        const char* e = getenv("MPCF_DEVICE");
        return e ? atoi(e) : 0;
    }

    void syncGPU() { check(mpcf_device_synchronize(current_device()), "GPU::syncGPU"); }
    void syncStream(streamID) { if (g_current) check(mpcf_synchronize(g_current), "GPU::syncStream"); }

    void tell_memUsage_GPU()
    {
        long long total_b = 0, free_b = 0;
        check(mpcf_device_info(current_device(), nullptr, 0, &total_b, &free_b, nullptr), "GPU::tell_memUsage_GPU");
        printf("=====================================================================\n");
        printf("[FREE MEMORY ON GPU  = %10.2f MB (%5.1f%%)]\n", free_b / 1048576.0, 100.0 * free_b / (double)total_b);
        printf("[USED MEMORY ON GPU  = %10.2f MB]\n", (total_b - free_b) / 1048576.0);
        printf("[TOTAL MEMORY ON GPU = %10.2f MB]\n", total_b / 1048576.0);
        printf("=====================================================================\n");
    }

    void tell_GPU()
    {
        char name[256];
        long long total_b = 0;
        int sms = 0;
        check(mpcf_device_info(current_device(), name, (int)sizeof(name), &total_b, nullptr, &sms), "GPU::tell_GPU");
        printf("[GPU %d: %s, %d SMs, %.1f GB]\n", current_device(), name, sms, total_b / 1e9);
    }
}
