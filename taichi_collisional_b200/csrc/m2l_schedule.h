// Generated by m2l_schedule in gen_swap_tables.py's cost model: degree sets per warp (4 warps),
// balanced by longest-processing-time on the per-degree FP64 instruction estimate.
#pragma once
template <int P> struct TcDegSets;
template <> struct TcDegSets<4> { static constexpr int L = 3; static constexpr int d[4][3] = {{4,-1,-1},{3,-1,-1},{2,-1,-1},{1,0,-1}}; };
template <> struct TcDegSets<6> { static constexpr int L = 3; static constexpr int d[4][3] = {{6,-1,-1},{5,0,-1},{4,1,-1},{3,2,-1}}; };
template <> struct TcDegSets<8> { static constexpr int L = 4; static constexpr int d[4][4] = {{8,1,-1,-1},{7,2,-1,-1},{6,3,-1,-1},{5,4,0,-1}}; };
template <> struct TcDegSets<10> { static constexpr int L = 4; static constexpr int d[4][4] = {{10,3,-1,-1},{9,4,0,-1},{8,5,1,-1},{7,6,2,-1}}; };
template <> struct TcDegSets<12> { static constexpr int L = 5; static constexpr int d[4][5] = {{12,5,1,0,-1},{11,6,2,-1,-1},{10,7,3,-1,-1},{9,8,4,-1,-1}}; };
template <> struct TcDegSets<16> { static constexpr int L = 6; static constexpr int d[4][6] = {{16,9,5,4,-1,-1},{15,10,6,3,-1,-1},{14,11,7,2,-1,-1},{13,12,8,1,0,-1}}; };
