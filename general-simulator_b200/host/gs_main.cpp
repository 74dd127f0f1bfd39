// gs_main.cpp -- gsi <script> [device]: run a General-Simulator script
// (src/main.cu:8-45).  The log goes to stdout and <script>.log.
#include <fstream>
#include <iterator>

#include "../../include/gs_capi.h"
#include "gs_driver.h"

int main(int argc, char** argv) {
  using namespace gsfe;
  std::string file;
  if (argc == 1) {
    file = "in.gs";
    log().open(file);
    log() << "Since no input script assigned, default \"in.gs\" is used.\n";
  } else {
    file = argv[1];
    log().open(file);
    log() << "Input script \"" << file << "\" is used.\n";
    if (argc == 3) {
      const int dev = std::atoi(argv[2]);
      gs_set_device(dev);
      log() << "Gpu device set to " << dev << "\n";
    }
  }
  std::ifstream in(file);
  if (!in) {
    log() << "Input script " << file << " is not found\n";
    return -1;
  }
  std::string script((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  Driver drv;
  Interpreter it(drv);
  Interpreter::standardize(script);
  it.run(script);
  log().flush();
  return 0;
}
