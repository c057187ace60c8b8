// Linked beside an unchanged reference application by tests/apps/Makefile.
// The reference's apps never check for errors (its library exits on them);
// this library records a code instead.  At exit, on the main thread that made
// every library call, the probe prints that code so a test can tell that all
// of the application's calls succeeded.
#include <cstdio>
#include <cstdlib>

extern "C" int vis_get_last_error(void);
extern "C" const char* vis_get_last_error_message(void);

namespace {

void report_last_error() {
    const char* msg = vis_get_last_error_message();
    std::printf("vis_get_last_error=%d (%s)\n", vis_get_last_error(), msg ? msg : "");
    std::fflush(stdout);
}

struct ExitProbe {
    ExitProbe() { std::atexit(report_last_error); }
} exit_probe;

}  // namespace
