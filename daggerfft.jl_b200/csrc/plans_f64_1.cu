// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<double,true,1024,2,1,2>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,2,1,2>(const PassDesc);
template __global__ void axis_pass_static<double,true,1024,9,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,9,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,9,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,9,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,20,4,5,4>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,20,4,5,4>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,20,4,5,4>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,20,4,5,4>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,36,6,6,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,36,6,6,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,36,6,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,36,6,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,60,6,10,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,60,6,10,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,60,6,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,60,6,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,90,6,15,6>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,90,6,15,6>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,90,6,15,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,90,6,15,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,128,8,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,128,8,16,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,128,8,16,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,128,8,16,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,180,12,15,12>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,180,12,15,12>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,180,12,15,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,180,12,15,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,243,81,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,243,81,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,4,243,81,3,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,243,81,3,3,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,320,40,5,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,320,40,5,8,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,320,40,5,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,320,40,5,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,512,405,27,15,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,405,27,15,3,3,3>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,405,27,15,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,405,27,15,3,3,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,512,64,8,8,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,512,64,8,8,8>(const PassDesc);
template __global__ void axis_pass_pipe<double,512,false,8,512,64,8,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<double,512,true,0,512,64,8,8,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<double,true,1024,648,108,6,6,6,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,648,108,6,6,6,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,800,80,10,10,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,800,80,10,10,8>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1000,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1000,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1215,81,15,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1215,81,15,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,1024,1458,243,6,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,false,1024,1458,243,6,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,1800,120,15,12,10>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,1800,120,15,12,10>(const PassDesc);
template __global__ void axis_pass_static<double,true,512,2048,128,16,16,8>(const PassDesc);
template __global__ void axis_pass_static<double,false,512,2048,128,16,16,8>(const PassDesc);
extern const StaticPlan kPlans_f64_1[];
extern const int kPlansCount_f64_1;
const StaticPlan kPlans_f64_1[] = {
  {2, 1, 1, {2}, 1024, (const void*)&axis_pass_static<double,true,1024,2,1,2>, (const void*)&axis_pass_static<double,false,1024,2,1,2>, nullptr, nullptr, 512, 0},
  {9, 3, 2, {3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,9,3,3,3>, (const void*)&axis_pass_static<double,false,1024,9,3,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,9,3,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,9,3,3,3>, 512, 8},
  {20, 4, 2, {5,4}, 1024, (const void*)&axis_pass_static<double,true,1024,20,4,5,4>, (const void*)&axis_pass_static<double,false,1024,20,4,5,4>, (const void*)&axis_pass_pipe<double,512,false,8,20,4,5,4>, (const void*)&axis_pass_pipe<double,512,true,0,20,4,5,4>, 512, 8},
  {36, 6, 2, {6,6}, 1024, (const void*)&axis_pass_static<double,true,1024,36,6,6,6>, (const void*)&axis_pass_static<double,false,1024,36,6,6,6>, (const void*)&axis_pass_pipe<double,512,false,8,36,6,6,6>, (const void*)&axis_pass_pipe<double,512,true,0,36,6,6,6>, 512, 8},
  {60, 6, 2, {10,6}, 512, (const void*)&axis_pass_static<double,true,512,60,6,10,6>, (const void*)&axis_pass_static<double,false,512,60,6,10,6>, (const void*)&axis_pass_pipe<double,512,false,8,60,6,10,6>, (const void*)&axis_pass_pipe<double,512,true,0,60,6,10,6>, 512, 8},
  {90, 6, 2, {15,6}, 512, (const void*)&axis_pass_static<double,true,512,90,6,15,6>, (const void*)&axis_pass_static<double,false,512,90,6,15,6>, (const void*)&axis_pass_pipe<double,512,false,8,90,6,15,6>, (const void*)&axis_pass_pipe<double,512,true,0,90,6,15,6>, 512, 8},
  {128, 8, 2, {16,8}, 512, (const void*)&axis_pass_static<double,true,512,128,8,16,8>, (const void*)&axis_pass_static<double,false,512,128,8,16,8>, (const void*)&axis_pass_pipe<double,512,false,8,128,8,16,8>, (const void*)&axis_pass_pipe<double,512,true,0,128,8,16,8>, 512, 8},
  {180, 12, 2, {15,12}, 512, (const void*)&axis_pass_static<double,true,512,180,12,15,12>, (const void*)&axis_pass_static<double,false,512,180,12,15,12>, (const void*)&axis_pass_pipe<double,512,false,8,180,12,15,12>, (const void*)&axis_pass_pipe<double,512,true,0,180,12,15,12>, 512, 8},
  {243, 81, 5, {3,3,3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,243,81,3,3,3,3,3>, (const void*)&axis_pass_static<double,false,1024,243,81,3,3,3,3,3>, (const void*)&axis_pass_pipe<double,512,false,4,243,81,3,3,3,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,243,81,3,3,3,3,3>, 512, 4},
  {320, 40, 3, {5,8,8}, 512, (const void*)&axis_pass_static<double,true,512,320,40,5,8,8>, (const void*)&axis_pass_static<double,false,512,320,40,5,8,8>, (const void*)&axis_pass_pipe<double,512,false,8,320,40,5,8,8>, (const void*)&axis_pass_pipe<double,512,true,0,320,40,5,8,8>, 512, 8},
  {405, 27, 4, {15,3,3,3}, 512, (const void*)&axis_pass_static<double,true,512,405,27,15,3,3,3>, (const void*)&axis_pass_static<double,false,512,405,27,15,3,3,3>, (const void*)&axis_pass_pipe<double,512,false,8,405,27,15,3,3,3>, (const void*)&axis_pass_pipe<double,512,true,0,405,27,15,3,3,3>, 512, 8},
  {512, 64, 3, {8,8,8}, 1024, (const void*)&axis_pass_static<double,true,1024,512,64,8,8,8>, (const void*)&axis_pass_static<double,false,1024,512,64,8,8,8>, (const void*)&axis_pass_pipe<double,512,false,8,512,64,8,8,8>, (const void*)&axis_pass_pipe<double,512,true,0,512,64,8,8,8>, 512, 8},
  {648, 108, 4, {6,6,6,3}, 1024, (const void*)&axis_pass_static<double,true,1024,648,108,6,6,6,3>, (const void*)&axis_pass_static<double,false,1024,648,108,6,6,6,3>, nullptr, nullptr, 512, 0},
  {800, 80, 3, {10,10,8}, 512, (const void*)&axis_pass_static<double,true,512,800,80,10,10,8>, (const void*)&axis_pass_static<double,false,512,800,80,10,10,8>, nullptr, nullptr, 512, 0},
  {1000, 100, 3, {10,10,10}, 512, (const void*)&axis_pass_static<double,true,512,1000,100,10,10,10>, (const void*)&axis_pass_static<double,false,512,1000,100,10,10,10>, nullptr, nullptr, 512, 0},
  {1215, 81, 5, {15,3,3,3,3}, 512, (const void*)&axis_pass_static<double,true,512,1215,81,15,3,3,3,3>, (const void*)&axis_pass_static<double,false,512,1215,81,15,3,3,3,3>, nullptr, nullptr, 512, 0},
  {1458, 243, 6, {6,3,3,3,3,3}, 1024, (const void*)&axis_pass_static<double,true,1024,1458,243,6,3,3,3,3,3>, (const void*)&axis_pass_static<double,false,1024,1458,243,6,3,3,3,3,3>, nullptr, nullptr, 512, 0},
  {1800, 120, 3, {15,12,10}, 512, (const void*)&axis_pass_static<double,true,512,1800,120,15,12,10>, (const void*)&axis_pass_static<double,false,512,1800,120,15,12,10>, nullptr, nullptr, 512, 0},
  {2048, 128, 3, {16,16,8}, 512, (const void*)&axis_pass_static<double,true,512,2048,128,16,16,8>, (const void*)&axis_pass_static<double,false,512,2048,128,16,16,8>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f64_1 = 19;
}  // namespace dfft
