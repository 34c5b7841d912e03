/* stand-in for OpenGraph's timer.h: wall-clock interval timer */
#ifndef REFSTUB_TIMER_H
#define REFSTUB_TIMER_H
#include <time.h>
struct Timer
{
    struct timespec start_time, end_time;
};
void Start(struct Timer *timer);
void Stop(struct Timer *timer);
double Seconds(struct Timer *timer);
#endif
