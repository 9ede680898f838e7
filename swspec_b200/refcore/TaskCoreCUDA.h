// TaskCoreCUDA.h -- the GPU core as a drop-in TaskCore of the reference.
//
// Derives from the reference's own abstract core (src/TaskCore.h:36-89) and
// takes the reference's settings struct (swspect_settings_t,
// src/Settings.h:59-159), so the reference's TaskDispatcher
// (src/TaskDispatcher.cpp:59-64, 92-247) drives it unchanged once
// TaskDispatcher.h selects it:
//
//   #elif defined(NVIDIA_CUDA)
//      #include "TaskCoreCUDA.h"
//      #define Platform_TaskCore TaskCoreCUDA
//
// Each method maps onto the C ABI of libswsgpu.so (include/swsgpu.h):
// prepare -> swsgpu_create, run -> swsgpu_submit (host-to-device copy and
// kernels queued, returns at once), join -> swsgpu_wait + swsgpu_fetch,
// finalize -> swsgpu_destroy.  combineResults adds a fetched run into the
// dispatcher's buffers, or, when the runs of one spectrum are summed on the
// device, copies the completed sum once.
#ifndef TASKCORECUDA_H
#define TASKCORECUDA_H

#include <cstdint>
#include <vector>

#include "Settings.h"
#include "TaskCore.h"
#include "swsgpu.h"

class TaskCoreCUDA : public TaskCore
{
public:
   explicit TaskCoreCUDA(int rank) : TaskCore(rank), rank_(rank) {}
   ~TaskCoreCUDA();

   void prepare(swspect_settings_t *settings);
   int run(Buffer **inbuf, Buffer **outbuf, Buffer **xpolbuf, Buffer **pcalbuf);
   int join();
   int finalize();
   int combineResults(Buffer **outbuf, Buffer **pcalbuf);
   void resetBuffer(Buffer *buf);

private:
   int rank_;
   swspect_settings_t *cfg_ = nullptr;
   swsgpu_handle *h_ = nullptr;
   Buffer **out_ = nullptr, **xpol_ = nullptr, **pcal_ = nullptr;
   int runs_per_output_ = 1;     // runs summed on the device per completed spectrum
   bool fetched_ = false;        // out_/xpol_/pcal_ hold spectra not yet combined
   int run_nspec_ = 0;
   int64_t runs_ = 0, ffts_ = 0;
   std::vector<float> staged_, stagedx_, stagedp_;
   std::vector<void *> pinned_;  // raw buffers page-locked for asynchronous input copies
};

#endif  // TASKCORECUDA_H
