// Command-line driver of a full run on the B200 path, with the reference's
// fluid_test interface (fluid_test.cc:10-32): reads <name>.cfg, writes the
// frames and restart files into <name>.odr, and with -r resumes from the last
// restart file there.
//
//   vdi_fluid_test [-r] <input_file.cfg>
#include <cstdio>
#include <cstring>
#include <sys/stat.h>

#include "fluid_2d.hh"

int main(int argc, char** argv) {
    bool resume = argc == 3 && strcmp(argv[1], "-r") == 0;
    if (argc != 2 && !resume) {
        fputs("Syntax: ./vdi_fluid_test [-r] <input_file>\n\n"
              "The input file should have a '.cfg' suffix\n", stderr);
        return 1;
    }
    fluid_2d f2d(argv[argc - 1]);
    mkdir(f2d.filename, S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH);
    if (resume) f2d.load_last_restart();
    else f2d.init_fields();
    f2d.solve();
    return 0;
}
