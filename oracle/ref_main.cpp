// `fluxos_ref <modset.json>`: the FLUXOS reference program built by
// oracle/Makefile (test infrastructure and the CPU baseline only).
extern "C" int fxr_main(const char* modset_path);
int main(int argc, char** argv) { return argc < 2 ? 2 : fxr_main(argv[1]); }
