// digholo_run: runs digHoloRunBatchFromConfigFile on every settings file
// named on the command line, as the reference's command-line program does
// (digHolo.cpp:17934-17943).
#include <cstdio>

extern "C" int digHoloRunBatchFromConfigFile(char* filename);

int main(int argc, char* argv[]) {
    int worst = 0;
    for (int i = 1; i < argc; i++) {
        printf("%d\t%s\n", i - 1, argv[i]);
        fflush(stdout);
        const int r = digHoloRunBatchFromConfigFile(argv[i]);
        if (r) worst = r;
    }
    return worst;
}
