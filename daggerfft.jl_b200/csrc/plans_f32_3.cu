// Generated by gen_plans.py -- do not edit.
#include "static_plans.h"
namespace dfft {
template __global__ void axis_pass_static<float,true,1024,4,1,4>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,4,1,4>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,12,1,12>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,12,1,12>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,12,1,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,12,1,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,25,5,5,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,25,5,5,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,45,3,15,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,45,3,15,3>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,45,3,15,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,45,3,15,3>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,72,6,12,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,72,6,12,6>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,72,6,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,72,6,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,100,10,10,10>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,100,10,10,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,100,10,10,10>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,144,12,12,12>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,144,12,12,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,144,12,12,12>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,200,25,5,5,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,200,25,5,5,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,200,25,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,200,25,5,5,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,256,16,16,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,256,16,16,16>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,256,16,16,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,256,16,16,16>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,360,36,10,6,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,360,36,10,6,6>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,360,36,10,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,360,36,10,6,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,450,30,15,6,5>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,450,30,15,6,5>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,16,450,30,15,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,450,30,15,6,5>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,576,48,12,6,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,576,48,12,6,8>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,16,576,48,12,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,576,48,12,6,8>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,720,60,12,10,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,720,60,12,10,6>(const PassDesc);
template __global__ void axis_pass_pipe<float,512,false,8,720,60,12,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,512,true,0,720,60,12,10,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,1024,864,72,12,12,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,864,72,12,12,6>(const PassDesc);
template __global__ void axis_pass_pipe<float,1024,false,8,864,72,12,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_pipe<float,1024,true,0,864,72,12,12,6>(const PassDesc, const __grid_constant__ CUtensorMap, const __grid_constant__ CUtensorMap, const TmaGeom);
template __global__ void axis_pass_static<float,true,512,1080,72,15,12,6>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,1080,72,15,12,6>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,1280,80,10,16,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,1280,80,10,16,8>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,1536,96,12,16,8>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,1536,96,12,16,8>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,1920,120,12,10,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,1920,120,12,10,16>(const PassDesc);
template __global__ void axis_pass_static<float,true,1024,2187,729,3,3,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,1024,2187,729,3,3,3,3,3,3,3>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,2560,160,10,16,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,2560,160,10,16,16>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,3072,192,12,16,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,3072,192,12,16,16>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,3600,225,15,15,16>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,3600,225,15,15,16>(const PassDesc);
template __global__ void axis_pass_static<float,true,512,4050,270,15,15,6,3>(const PassDesc);
template __global__ void axis_pass_static<float,false,512,4050,270,15,15,6,3>(const PassDesc);
extern const StaticPlan kPlans_f32_3[];
extern const int kPlansCount_f32_3;
const StaticPlan kPlans_f32_3[] = {
  {4, 1, 1, {4}, 1024, (const void*)&axis_pass_static<float,true,1024,4,1,4>, (const void*)&axis_pass_static<float,false,1024,4,1,4>, nullptr, nullptr, 1024, 0},
  {12, 1, 1, {12}, 1024, (const void*)&axis_pass_static<float,true,1024,12,1,12>, (const void*)&axis_pass_static<float,false,1024,12,1,12>, (const void*)&axis_pass_pipe<float,1024,false,16,12,1,12>, (const void*)&axis_pass_pipe<float,1024,true,0,12,1,12>, 1024, 16},
  {25, 5, 2, {5,5}, 1024, (const void*)&axis_pass_static<float,true,1024,25,5,5,5>, (const void*)&axis_pass_static<float,false,1024,25,5,5,5>, (const void*)&axis_pass_pipe<float,1024,false,16,25,5,5,5>, (const void*)&axis_pass_pipe<float,1024,true,0,25,5,5,5>, 1024, 16},
  {45, 3, 2, {15,3}, 1024, (const void*)&axis_pass_static<float,true,1024,45,3,15,3>, (const void*)&axis_pass_static<float,false,1024,45,3,15,3>, (const void*)&axis_pass_pipe<float,1024,false,16,45,3,15,3>, (const void*)&axis_pass_pipe<float,1024,true,0,45,3,15,3>, 1024, 16},
  {72, 6, 2, {12,6}, 1024, (const void*)&axis_pass_static<float,true,1024,72,6,12,6>, (const void*)&axis_pass_static<float,false,1024,72,6,12,6>, (const void*)&axis_pass_pipe<float,1024,false,16,72,6,12,6>, (const void*)&axis_pass_pipe<float,1024,true,0,72,6,12,6>, 1024, 16},
  {100, 10, 2, {10,10}, 1024, (const void*)&axis_pass_static<float,true,1024,100,10,10,10>, (const void*)&axis_pass_static<float,false,1024,100,10,10,10>, (const void*)&axis_pass_pipe<float,1024,false,16,100,10,10,10>, (const void*)&axis_pass_pipe<float,1024,true,0,100,10,10,10>, 1024, 16},
  {144, 12, 2, {12,12}, 1024, (const void*)&axis_pass_static<float,true,1024,144,12,12,12>, (const void*)&axis_pass_static<float,false,1024,144,12,12,12>, (const void*)&axis_pass_pipe<float,1024,false,16,144,12,12,12>, (const void*)&axis_pass_pipe<float,1024,true,0,144,12,12,12>, 1024, 16},
  {200, 25, 3, {5,5,8}, 1024, (const void*)&axis_pass_static<float,true,1024,200,25,5,5,8>, (const void*)&axis_pass_static<float,false,1024,200,25,5,5,8>, (const void*)&axis_pass_pipe<float,1024,false,16,200,25,5,5,8>, (const void*)&axis_pass_pipe<float,1024,true,0,200,25,5,5,8>, 1024, 16},
  {256, 16, 2, {16,16}, 1024, (const void*)&axis_pass_static<float,true,1024,256,16,16,16>, (const void*)&axis_pass_static<float,false,1024,256,16,16,16>, (const void*)&axis_pass_pipe<float,1024,false,16,256,16,16,16>, (const void*)&axis_pass_pipe<float,1024,true,0,256,16,16,16>, 1024, 16},
  {360, 36, 3, {10,6,6}, 1024, (const void*)&axis_pass_static<float,true,1024,360,36,10,6,6>, (const void*)&axis_pass_static<float,false,1024,360,36,10,6,6>, (const void*)&axis_pass_pipe<float,1024,false,16,360,36,10,6,6>, (const void*)&axis_pass_pipe<float,1024,true,0,360,36,10,6,6>, 1024, 16},
  {450, 30, 3, {15,6,5}, 512, (const void*)&axis_pass_static<float,true,512,450,30,15,6,5>, (const void*)&axis_pass_static<float,false,512,450,30,15,6,5>, (const void*)&axis_pass_pipe<float,512,false,16,450,30,15,6,5>, (const void*)&axis_pass_pipe<float,512,true,0,450,30,15,6,5>, 512, 16},
  {576, 48, 3, {12,6,8}, 1024, (const void*)&axis_pass_static<float,true,1024,576,48,12,6,8>, (const void*)&axis_pass_static<float,false,1024,576,48,12,6,8>, (const void*)&axis_pass_pipe<float,1024,false,16,576,48,12,6,8>, (const void*)&axis_pass_pipe<float,1024,true,0,576,48,12,6,8>, 1024, 16},
  {720, 60, 3, {12,10,6}, 512, (const void*)&axis_pass_static<float,true,512,720,60,12,10,6>, (const void*)&axis_pass_static<float,false,512,720,60,12,10,6>, (const void*)&axis_pass_pipe<float,512,false,8,720,60,12,10,6>, (const void*)&axis_pass_pipe<float,512,true,0,720,60,12,10,6>, 512, 8},
  {864, 72, 3, {12,12,6}, 1024, (const void*)&axis_pass_static<float,true,1024,864,72,12,12,6>, (const void*)&axis_pass_static<float,false,1024,864,72,12,12,6>, (const void*)&axis_pass_pipe<float,1024,false,8,864,72,12,12,6>, (const void*)&axis_pass_pipe<float,1024,true,0,864,72,12,12,6>, 1024, 8},
  {1080, 72, 3, {15,12,6}, 512, (const void*)&axis_pass_static<float,true,512,1080,72,15,12,6>, (const void*)&axis_pass_static<float,false,512,1080,72,15,12,6>, nullptr, nullptr, 512, 0},
  {1280, 80, 3, {10,16,8}, 512, (const void*)&axis_pass_static<float,true,512,1280,80,10,16,8>, (const void*)&axis_pass_static<float,false,512,1280,80,10,16,8>, nullptr, nullptr, 512, 0},
  {1536, 96, 3, {12,16,8}, 512, (const void*)&axis_pass_static<float,true,512,1536,96,12,16,8>, (const void*)&axis_pass_static<float,false,512,1536,96,12,16,8>, nullptr, nullptr, 512, 0},
  {1920, 120, 3, {12,10,16}, 512, (const void*)&axis_pass_static<float,true,512,1920,120,12,10,16>, (const void*)&axis_pass_static<float,false,512,1920,120,12,10,16>, nullptr, nullptr, 512, 0},
  {2187, 729, 7, {3,3,3,3,3,3,3}, 1024, (const void*)&axis_pass_static<float,true,1024,2187,729,3,3,3,3,3,3,3>, (const void*)&axis_pass_static<float,false,1024,2187,729,3,3,3,3,3,3,3>, nullptr, nullptr, 1024, 0},
  {2560, 160, 3, {10,16,16}, 512, (const void*)&axis_pass_static<float,true,512,2560,160,10,16,16>, (const void*)&axis_pass_static<float,false,512,2560,160,10,16,16>, nullptr, nullptr, 512, 0},
  {3072, 192, 3, {12,16,16}, 512, (const void*)&axis_pass_static<float,true,512,3072,192,12,16,16>, (const void*)&axis_pass_static<float,false,512,3072,192,12,16,16>, nullptr, nullptr, 512, 0},
  {3600, 225, 3, {15,15,16}, 512, (const void*)&axis_pass_static<float,true,512,3600,225,15,15,16>, (const void*)&axis_pass_static<float,false,512,3600,225,15,15,16>, nullptr, nullptr, 512, 0},
  {4050, 270, 4, {15,15,6,3}, 512, (const void*)&axis_pass_static<float,true,512,4050,270,15,15,6,3>, (const void*)&axis_pass_static<float,false,512,4050,270,15,15,6,3>, nullptr, nullptr, 512, 0},
};
const int kPlansCount_f32_3 = 23;
}  // namespace dfft
