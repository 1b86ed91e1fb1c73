// Prints n -> CGenMathFFT::NextCorrectNumberForFFT(n) from the reference's own gmfft.cpp, as runs
// "first_n last_n result" (test infrastructure: pins the good-number table of the oracle).
#include <cstdio>
#include <cstdlib>
#include "gmfft.h"
int main(int argc, char** argv)
{
	long nmax = (argc > 1) ? atol(argv[1]) : 300000;
	CGenMathFFT fft;
	long runStart = 1, prev = -1;
	for(long n = 1; n <= nmax; n++)
	{
		long m = n; fft.NextCorrectNumberForFFT(m);
		if(m != prev)
		{
			if(prev >= 0) printf("%ld %ld %ld\n", runStart, n - 1, prev);
			runStart = n; prev = m;
		}
	}
	printf("%ld %ld %ld\n", runStart, nmax, prev);
	return 0;
}
