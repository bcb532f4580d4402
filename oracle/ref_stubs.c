/* ref_stubs.c -- test infrastructure, not product code.
 *
 * The reference's `galn` binary dispatches four subcommands from one main() (galn.cu:1294-1304).
 * oracle/Makefile builds it from the reference's own aln sources only (galn.cu, host_io.c, aln_host.c,
 * aln_il.c), so the index/samse/sampe entry points it names are provided here as stubs that refuse to
 * run. `galn_ref aln ...` is then the reference's unmodified aln command, used as the parity oracle and
 * as the timed CPU baseline.
 */
#include <stdio.h>

static int not_built(const char *what)
{
    fprintf(stderr, "[galn_ref] '%s' is not part of this oracle build (aln only)\n", what);
    return 1;
}

int galn_index(int argc, char *argv[]) { (void)argc; (void)argv; return not_built("index"); }
int galn_samse(int argc, char *argv[]) { (void)argc; (void)argv; return not_built("samse"); }
int galn_sampe(int argc, char *argv[]) { (void)argc; (void)argv; return not_built("sampe"); }
