/*
 * dropin_lumcolumn.c -- the one function a maintainer adds to run lu2's own
 * main (lu2.c:1220-1309) on the GPU library: lu2.c is compiled with
 * -Dlumcolumn=lumcolumn_cpu (its definition and main's call both renamed)
 * and that definition is made weak (objcopy --weaken-symbol=lumcolumn_cpu),
 * so main's call binds to this strong definition, which forwards to
 * liblu2gpu.so's lumcolumn (lu2.c:1122 signature).
 *
 * TEST INFRASTRUCTURE: built by oracle/build_oracle.py into oracle/_ref/
 * (the executable lu2_gpu); never part of the library.
 */
void lumcolumn(int n, double *a, double *b, int m, double *awork, int *pv, int recursive);

void lumcolumn_cpu(int n, double *a, double *b, int m, double *awork, int *pv, int recursive)
{
    lumcolumn(n, a, b, m, awork, pv, recursive);
}
