// Prints a small tensor with printTensor (inc/cudecompose.h of
// 891922758/first-project).  Built once against this repository's drop-in
// archive and once against the reference library, the two outputs must be
// identical (the debug print's layout is src/kr.cu:13-30).
#include "cudecompose.h"

int main() {
    const long a = 3, b = 2, c = 2;
    float h[12];
    for (int i = 0; i < 12; i++) h[i] = 0.25f * (float)(i * i) - 3.0f + (i % 3 == 0 ? 1e-3f * (float)i : 0.0f);
    float *d;
    cudaMalloc((void **)&d, sizeof(h));
    cudaMemcpy(d, h, sizeof(h), cudaMemcpyHostToDevice);
    printTensor(d, a, b, c);
    cudaFree(d);
    return 0;
}
