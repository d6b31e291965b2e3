/* A C host of tenes_gpu_main: loads libtenes_gpu.so, runs each input file
 * given on the command line in order, prints the status of every call, and
 * exits with the last status.  The process has no Python of its own, so the
 * library brings up its embedded interpreter on the first call. */
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s <libtenes_gpu.so> <print_level> <input.toml>...\n", argv[0]);
    return 100;
  }
  void* h = dlopen(argv[1], RTLD_NOW);
  if (!h) {
    fprintf(stderr, "dlopen: %s\n", dlerror());
    return 101;
  }
  int (*run)(const char*, int) = (int (*)(const char*, int))dlsym(h, "tenes_gpu_main");
  const char* (*last_error)(void) = (const char* (*)(void))dlsym(h, "tg_last_error");
  if (!run || !last_error) {
    fprintf(stderr, "missing symbol\n");
    return 102;
  }
  int rc = 0;
  for (int i = 3; i < argc; ++i) {
    rc = run(argv[i], atoi(argv[2]));
    printf("status %d\n", rc);
    if (rc != 0) printf("message %s\n", last_error());
    fflush(stdout);
  }
  return rc;
}
