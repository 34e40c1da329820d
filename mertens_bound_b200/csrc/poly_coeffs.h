// Generated by gen_poly.py -- polynomial coefficients fitted by Chebyshev interpolation.
// Ascending powers of u = t^2; see gen_poly.py for the meaning of each set.
#pragma once
// HALF_S: degree 8 in u, max rel. fit error 3.23e-19
static __device__ __constant__ const double HALF_S[9] = {3.141592653589793, -5.167712780049969, 2.5501640398773007, -0.5992645293189447, 0.0821458865731029, -0.007370430505916944, 0.0004662998161898394, -2.1903497074626018e-05, 7.697826768224191e-07};
// HALF_C: degree 9 in u, max abs. fit error 6.38e-21
static __device__ __constant__ const double HALF_C[10] = {1.0, -4.934802200544679, 4.058712126416768, -1.3352627688545549, 0.235330630357995, -0.025806891376592964, 0.0019295741872812349, -0.00010463741681752138, 4.300724172734847e-06, -1.34352129509532e-07};
// QUAD_S: degree 5 in u, max rel. fit error 4.74e-15
static __device__ __constant__ const double QUAD_S[6] = {6.28318530717956, -41.34170224027578, 81.60524918348393, -76.70583445845129, 42.05556925594499, -14.916565118819118};
// QUAD_C: degree 5 in u, max abs. fit error 5.56e-14
static __device__ __constant__ const double QUAD_C[6] = {0.9999999999999444, -19.739208801922548, 64.93939383134831, -85.45676493719407, 60.23818359301454, -26.058123753882793};
// F32_S: degree 3 in u, max rel. fit error 3.4e-9
static __device__ __constant__ const float F32_S[4] = {6.2831854820251465f, -41.3416633605957f, 81.59254455566406f, -75.401611328125f};
// F32_C: degree 4 in u, max abs. fit error 4.75e-11
static __device__ __constant__ const float F32_C[5] = {1.0f, -19.739208221435547f, 64.93931579589844f, -85.4428482055664f, 59.22016906738281f};
