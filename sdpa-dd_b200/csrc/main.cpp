// sdpa_dd_b200: drop-in for the reference's sdpa_dd command.
#include "../../include/sddd.h"
int main(int argc, char **argv) { return sddd_cli_main(argc, argv); }
