// ref_serial_scheduler.cpp — the shim runs the reference's code without a task scheduler (test
// infrastructure only, linked into oracle/_ref/libsdx_ref.so by oracle/build_ref.sh).
//
// The reference's BlockSparseMatrix::Apply and BlockJacobiPrec look up mochi::TaskScheduler::TryGet()
// (mochi_core/include/mochi_core/utils/task_scheduler.h:110) and run serially when it returns null, which
// is the reference's own single-threaded configuration. The scheduler itself (task_scheduler.cpp, built
// on the vendored marl library) is not compiled here: TryGet() returns null, and the members that only a
// live scheduler reaches abort if they are ever called.
#include <mochi_core/utils/task_scheduler.h>

#include <cstdlib>

namespace mochi {

TaskScheduler* TaskScheduler::TryGet() { return nullptr; }
int TaskScheduler::GetNumOtherThreads() const { std::abort(); }
void TaskScheduler::AddTaskNoProfile(TaskFn&&, bool) { std::abort(); }
void TaskScheduler::TryToWakeUpMoreWorkers(int, TimeSpan) { std::abort(); }
TaskSemaphore::TaskSemaphore(int) { std::abort(); }
void TaskSemaphore::Add(int) const { std::abort(); }
bool TaskSemaphore::Done(int) const { std::abort(); }
void TaskSemaphore::Wait() const { std::abort(); }

}  // namespace mochi
