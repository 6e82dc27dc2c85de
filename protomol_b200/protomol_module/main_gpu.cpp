// ProtoMol's command-line driver with the GPU force module added to the
// stock module set (the same steps as the reference's main.cpp).
#include <protomol/ProtoMolApp.h>
#include <protomol/base/Exception.h>
#include <protomol/base/ModuleManager.h>

#include <iostream>

#include "PmgpuForceModule.h"

using namespace std;
using namespace ProtoMol;

extern void moduleInitFunction(ModuleManager *);

int main(int argc, char *argv[]) {
  try {
    ModuleManager modManager;
    moduleInitFunction(&modManager);
    modManager.add(new PmgpuForceModule());
    ProtoMolApp app(&modManager);
    if (!app.configure(argc, argv)) return 0;
    app.splash(cout);
    app.build();
    while (app.step()) continue;
    app.finalize();
    return 0;
  } catch (const Exception &e) {
    cerr << "ERROR: " << e << endl;
  }
  return 1;
}
