// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<double,true,1024,5,1,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,5,1,5>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,15,1,15>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,15,1,15>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,15,1,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,15,1,15>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,27,9,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,27,9,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,27,9,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,27,9,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,48,6,6,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,48,6,6,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,48,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,48,6,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,75,5,15,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,75,5,15,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,75,5,15,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,75,5,15,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,108,18,6,6,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,108,18,6,6,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,108,18,6,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,108,18,6,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,150,10,15,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,150,10,15,10>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,150,10,15,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,150,10,15,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,216,36,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,216,36,6,6,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,216,36,6,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,216,36,6,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,270,18,15,6,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,270,18,15,6,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,270,18,15,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,270,18,15,6,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,375,25,15,5,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,375,25,15,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,375,25,15,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,375,25,15,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,480,48,10,6,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,480,48,10,6,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,480,48,10,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,480,48,10,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,600,60,10,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,600,60,10,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,1024,729,243,3,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,729,243,3,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,900,60,15,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,900,60,15,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1125,75,15,15,5>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1125,75,15,15,5>(const PassDesc);
template __global__ void axis_pass_static<double,true,1024,1296,216,6,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,1296,216,6,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1600,100,10,10,16>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1600,100,10,10,16>(const PassDesc);
template __global__ void axis_pass_static<double,true,1024,1944,324,6,6,6,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,1944,324,6,6,6,3,3>(const PassDesc);
extern const StaticPlan kPlans_f64_4[];
extern const int kPlansCount_f64_4;
const StaticPlan kPlans_f64_4[] = {
  {5, 1, 1, {5}, 1024, (const void*)&axis_pass_static<double,true,1024,5,1,5>, (const void*)&axis_pass_static<double,false,1024,5,1,5>, nullptr, nullptr, 512, 0},
  {15, 1, 1, {15}, 512, (const void*)&axis_pass_static<double,true,512,15,1,15>, (const void*)&axis_pass_static<double,false,512,15,1,15>, (const void*)&axis_pass_pipe<double,512,false,8,15,1,15>, (const void*)&axis_pass_pipe<double,512,true,0,15,1,15>, 512, 8},
  {27, 9, 3, {3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,27,9,3,3,3>, (const void*)&axis_pass_static<double,false,1024,27,9,3,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,27,9,3,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,27,9,3,3,3>, 512, 8},
  {48, 6, 2, {6,8}, 512, (const void*)&axis_pass_static<double,true,512,48,6,6,8>, (const void*)&axis_pass_static<double,false,512,48,6,6,8>, (const void*)&axis_pass_pipe<double,512,false,8,48,6,6,8>, (const void*)&axis_pass_pipe<double,512,true,0,48,6,6,8>, 512, 8},
  {75, 5, 2, {15,5}, 512, (const void*)&axis_pass_static<double,true,512,75,5,15,5>, (const void*)&axis_pass_static<double,false,512,75,5,15,5>, (const void*)&axis_pass_pipe<double,512,false,8,75,5,15,5>, (const void*)&axis_pass_pipe<double,512,true,0,75,5,15,5>, 512, 8},
  {108, 18, 3, {6,6,3}, 1024, (const void*)&axis_pass_static<double,true,1024,108,18,6,6,3>, (const void*)&axis_pass_static<double,false,1024,108,18,6,6,3>, (const void*)&axis_pass_pipe<double,512,false,8,108,18,6,6,3>, (const void*)&axis_pass_pipe<double,512,true,0,108,18,6,6,3>, 512, 8},
  {150, 10, 2, {15,10}, 512, (const void*)&axis_pass_static<double,true,512,150,10,15,10>, (const void*)&axis_pass_static<double,false,512,150,10,15,10>, (const void*)&axis_pass_pipe<double,512,false,8,150,10,15,10>, (const void*)&axis_pass_pipe<double,512,true,0,150,10,15,10>, 512, 8},
  {216, 36, 3, {6,6,6}, 1024, (const void*)&axis_pass_static<double,true,1024,216,36,6,6,6>, (const void*)&axis_pass_static<double,false,1024,216,36,6,6,6>, (const void*)&axis_pass_pipe<double,512,false,8,216,36,6,6,6>, (const void*)&axis_pass_pipe<double,512,true,0,216,36,6,6,6>, 512, 8},
  {270, 18, 3, {15,6,3}, 512, (const void*)&axis_pass_static<double,true,512,270,18,15,6,3>, (const void*)&axis_pass_static<double,false,512,270,18,15,6,3>, (const void*)&axis_pass_pipe<double,512,false,8,270,18,15,6,3>, (const void*)&axis_pass_pipe<double,512,true,0,270,18,15,6,3>, 512, 8},
  {375, 25, 3, {15,5,5}, 512, (const void*)&axis_pass_static<double,true,512,375,25,15,5,5>, (const void*)&axis_pass_static<double,false,512,375,25,15,5,5>, (const void*)&axis_pass_pipe<double,512,false,8,375,25,15,5,5>, (const void*)&axis_pass_pipe<double,512,true,0,375,25,15,5,5>, 512, 8},
  {480, 48, 3, {10,6,8}, 512, (const void*)&axis_pass_static<double,true,512,480,48,10,6,8>, (const void*)&axis_pass_static<double,false,512,480,48,10,6,8>, (const void*)&axis_pass_pipe<double,512,false,8,480,48,10,6,8>, (const void*)&axis_pass_pipe<double,512,true,0,480,48,10,6,8>, 512, 8},
  {600, 60, 3, {10,10,6}, 512, (const void*)&axis_pass_static<double,true,512,600,60,10,10,6>, (const void*)&axis_pass_static<double,false,512,600,60,10,10,6>, nullptr, nullptr, 512, 0},
  {729, 243, 6, {3,3,3,3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,729,243,3,3,3,3,3,3>, (const void*)&axis_pass_static<double,false,1024,729,243,3,3,3,3,3,3>, nullptr, nullptr, 512, 0},
  {900, 60, 3, {15,10,6}, 512, (const void*)&axis_pass_static<double,true,512,900,60,15,10,6>, (const void*)&axis_pass_static<double,false,512,900,60,15,10,6>, nullptr, nullptr, 512, 0},
  {1125, 75, 3, {15,15,5}, 512, (const void*)&axis_pass_static<double,true,512,1125,75,15,15,5>, (const void*)&axis_pass_static<double,false,512,1125,75,15,15,5>, nullptr, nullptr, 512, 0},
  {1296, 216, 4, {6,6,6,6}, 1024, (const void*)&axis_pass_static<double,true,1024,1296,216,6,6,6,6>, (const void*)&axis_pass_static<double,false,1024,1296,216,6,6,6,6>, nullptr, nullptr, 512, 0},
  {1600, 100, 3, {10,10,16}, 512, (const void*)&axis_pass_static<double,true,512,1600,100,10,10,16>, (const void*)&axis_pass_static<double,false,512,1600,100,10,10,16>, nullptr, nullptr, 512, 0},
  {1944, 324, 5, {6,6,6,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,1944,324,6,6,6,3,3>, (const void*)&axis_pass_static<double,false,1024,1944,324,6,6,6,3,3>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f64_4 = 18;
}  // namespace dfft
