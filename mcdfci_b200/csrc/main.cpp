// mcdfci: command-line driver with the reference's usage (src/main.cpp:19-36):
//   mcdfci input.json
// reads the JSON input deck and the FCIDUMP it names, prints the report
// table and exits 0, or prints "ERROR: ..." and exits 1.
#include "../../include/mcdfci.h"

int main(int argc, char* argv[]) { return mcd_run_json(argc < 2 ? nullptr : argv[1]); }
